// HP-1: one fused kernel per low-storage RK3 stage.
//
// The reference (src/dg/explicit.c:75-96) does, per stage i:
//   dg_update_boundary(t + C_i dt); temp = F w; dw = M^-1 temp;
//   k2 = A_i k2 - dt dw; w += B_i k2
// with F and M^-1 assembled as global CSR matrices (simulation.c:218-491).
// Here the same operator is applied matrix-free, element by element:
//   R = (curl H, -curl E)          volume: -sum_j A(c_ij) w_j with
//                                  c_ij = codtau . int d(phi_i) phi_j
//                                  (simulation.c:263-324), so the physical
//                                  derivative of a field is codtau applied to
//                                  the three reference derivatives D_k w
//     + sum_faces S F_upwind(w_own, w_nb, vn)   (simulation.c:356-491)
//   dw = (1/det) Minv R            (simulation.c:241-243)
// Face fluxes are computed by each element with its own outward normal; the
// upwind flux is antisymmetric under (wL, wR, n) -> (wR, wL, -n), so this is
// the reference's +/- pair up to rounding.  Boundary neighbours read the
// analytic data at the face-node coordinates and the stage time
// (dg_update_boundary, dg.c:76-106), written by boundary_trace_kernel just
// before the stage.
//
// Work decomposition (TE = 32 elements per CTA, 6 warps):
//   A  16-byte coalesced loads of the tile (w, k2, geometry, neighbours) into
//      shared memory, transposed to [value][element] with stride TE+1 so that
//      lane = element is conflict-free everywhere below;
//   B  flux: warp w evaluates face-node slots {w, w+6, w+12, w+18} of its 32
//      elements (warp-uniform face / node);
//   C  volume: warp c owns field c; the 10 nodal values stay in registers,
//      r_k = D_k w_c with the tables as constant-bank FMA operands and the P2
//      structural zeros removed at compile time; only the two physical
//      derivatives the curl needs are written out (20 values);
//   D  warp c assembles R_c = curl part + sum_faces S F_c, lifts with Minv
//      (registers) and applies the RK update;
//   E  16-byte coalesced stores.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace gdn {

// Structural nonzeros of int d_k(phi_i) phi_j for the P2 basis (bit j of
// row i), and of the P2 triangle mass.  Checked against the tables at attach
// (entries outside the pattern must be below 1e-15 in magnitude).
__host__ __device__ constexpr unsigned dmask(int k, int i)
{
	constexpr unsigned short m[3][10] = {{0x3ff, 0x3ff, 0x000, 0x000, 0x1e3, 0x3fb, 0x3fb, 0x3f7, 0x3f7, 0x000},
										 {0x3ff, 0x000, 0x3ff, 0x000, 0x3fd, 0x3fd, 0x2b5, 0x3f7, 0x000, 0x3f7},
										 {0x3ff, 0x000, 0x000, 0x3ff, 0x3fd, 0x000, 0x3fb, 0x359, 0x3fd, 0x3fb}};
	return m[k][i];
}
__host__ __device__ constexpr unsigned smask(int i)
{
	constexpr unsigned char m[6] = {0x17, 0x27, 0x0f, 0x3c, 0x39, 0x3a};
	return m[i];
}
// the reference's P2 face-node convention (t10.c:37-42)
__host__ __device__ constexpr int f2n(int f, int j)
{
	constexpr int m[4][6] = {{0, 3, 2, 7, 9, 6}, {0, 1, 3, 4, 8, 7}, {0, 2, 1, 6, 5, 4}, {1, 2, 3, 5, 9, 8}};
	return m[f][j];
}

// r[k][i] = sum_j D_k[i][j] w[j] for the three reference directions, with the
// structural zeros skipped at compile time.
template <typename T, bool SPARSE>
__device__ __forceinline__ void ref_derivatives(const Tables<T> &tb, const T w[10], T r[3][10])
{
#pragma unroll
	for (int k = 0; k < 3; k++)
#pragma unroll
		for (int i = 0; i < 10; i++) {
			T acc = T(0);
#pragma unroll
			for (int j = 0; j < 10; j++)
				if (!SPARSE || (dmask(k, i) >> j & 1))
					acc += tb.D[k][i][j] * w[j];
			r[k][i] = acc;
		}
}

// FP32: the same sums with Blackwell's packed FP32x2 FMA, pairing
// (r0[i], r1[i]) and (r2[2m], r2[2m+1]); coefficient pairs are stored
// adjacent in constant memory (Tables<float>::D01, D2p).
template <>
__device__ __forceinline__ void ref_derivatives<float, true>(const Tables<float> &tb, const float w[10],
															 float r[3][10])
{
	float2 p01[10], p2[5];
#pragma unroll
	for (int i = 0; i < 10; i++)
		p01[i] = make_float2(0.f, 0.f);
#pragma unroll
	for (int m = 0; m < 5; m++)
		p2[m] = make_float2(0.f, 0.f);
#pragma unroll
	for (int j = 0; j < 10; j++) {
		const float2 wd = make_float2(w[j], w[j]);
#pragma unroll
		for (int i = 0; i < 10; i++)
			if ((dmask(0, i) | dmask(1, i)) >> j & 1)
				p01[i] = __ffma2_rn(tb.D01[i][j], wd, p01[i]);
#pragma unroll
		for (int m = 0; m < 5; m++)
			if ((dmask(2, 2 * m) | dmask(2, 2 * m + 1)) >> j & 1)
				p2[m] = __ffma2_rn(tb.D2p[m][j], wd, p2[m]);
	}
#pragma unroll
	for (int i = 0; i < 10; i++) {
		r[0][i] = p01[i].x;
		r[1][i] = p01[i].y;
	}
#pragma unroll
	for (int m = 0; m < 5; m++) {
		r[2][2 * m] = p2[m].x;
		r[2][2 * m + 1] = p2[m].y;
	}
}

// dw = Minv R (dense 10 x 10)
template <typename T>
__device__ __forceinline__ void lift_minv(const Tables<T> &tb, const T R[10], T dw[10])
{
#pragma unroll
	for (int i = 0; i < 10; i++) {
		T acc = T(0);
#pragma unroll
		for (int j = 0; j < 10; j++)
			acc += tb.Minv[i][j] * R[j];
		dw[i] = acc;
	}
}

template <>
__device__ __forceinline__ void lift_minv<float>(const Tables<float> &tb, const float R[10], float dw[10])
{
	float2 acc[5];
#pragma unroll
	for (int m = 0; m < 5; m++)
		acc[m] = make_float2(0.f, 0.f);
#pragma unroll
	for (int j = 0; j < 10; j++) {
		const float2 rd = make_float2(R[j], R[j]);
#pragma unroll
		for (int m = 0; m < 5; m++)
			acc[m] = __ffma2_rn(tb.MinvP[m][j], rd, acc[m]);
	}
#pragma unroll
	for (int m = 0; m < 5; m++) {
		dw[2 * m] = acc[m].x;
		dw[2 * m + 1] = acc[m].y;
	}
}

constexpr int kRk3Tile = 32; // elements per CTA
constexpr int kRk3Threads = 192; // 6 warps

template <typename T>
struct Rk3Smem {
	static constexpr int P = kRk3Tile + 1;
	// sW 60, sK 60, sF 144, sX 120, sG 10 rows of P values; then 8 ints per element
	static constexpr int rows = 60 + 60 + 144 + 120 + 10;
	static constexpr int bytes = rows * P * (int)sizeof(T) + 8 * kRk3Tile * (int)sizeof(int);
};

template <typename T, bool SPARSE>
__global__ void __launch_bounds__(kRk3Threads) rk3_stage_kernel(Rk3Params<T> p)
{
	constexpr int TE = kRk3Tile, P = Rk3Smem<T>::P;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T *sW = reinterpret_cast<T *>(smem_raw); // [60][P]   value k = node*6 + field
	T *sK = sW + 60 * P; // [60][P]
	T *sF = sK + 60 * P; // [144][P]  (face*6 + jj)*6 + c
	T *sX = sF + 144 * P; // [120][P]  (field*2 + which)*10 + node
	T *sG = sX + 120 * P; // [10][P]   codtau row-major, det
	int *sNb = reinterpret_cast<int *>(sG + 10 * P); // [TE][4]
	int *sPm = sNb + 4 * TE; // [TE][4]

	const Tables<T> &tb = tab<T>();
	const int tid = threadIdx.x;
	const int warp = tid >> 5, lane = tid & 31;
	const long long e0 = (long long)blockIdx.x * TE;
	const int nloc = (int)min((long long)TE, p.ne - e0);

	// ---- A: stage the tile ----
	{
		constexpr int VPC = 16 / sizeof(T);
		const int nch = nloc * 60 / VPC;
		const uint4 *gw = reinterpret_cast<const uint4 *>(p.w_in + e0 * 60);
		const uint4 *gk = reinterpret_cast<const uint4 *>(p.k2 + e0 * 60);
		for (int ch = tid; ch < nch; ch += kRk3Threads) {
			const int v0 = ch * VPC;
			const int e = v0 / 60, k = v0 % 60;
			const uint4 a = __ldg(gw + ch);
			const T *av = reinterpret_cast<const T *>(&a);
#pragma unroll
			for (int q = 0; q < VPC; q++)
				sW[(k + q) * P + e] = av[q];
		}
		if (!p.stage0) {
			for (int ch = tid; ch < nch; ch += kRk3Threads) {
				const int v0 = ch * VPC;
				const int e = v0 / 60, k = v0 % 60;
				const uint4 b = __ldcs(gk + ch);
				const T *bv = reinterpret_cast<const T *>(&b);
#pragma unroll
				for (int q = 0; q < VPC; q++)
					sK[(k + q) * P + e] = bv[q];
			}
		}
		for (int v = tid; v < nloc * 10; v += kRk3Threads)
			sG[(v % 10) * P + v / 10] = p.geom[e0 * 10 + v];
		if (tid < nloc * 4) {
			sNb[tid] = p.nb[e0 * 4 + tid];
			sPm[tid] = p.perm[e0 * 4 + tid];
		}
	}
	__syncthreads();

	const int e = lane;
	const bool live = e < nloc;

	// out-of-tile neighbour traces (or boundary data at the stage time) of this
	// thread's flux slots -- face node jj = warp of faces 0..3 -- issued now
	// and consumed after the volume phase, which hides their latency
	T pre[4][6];
	if (live) {
		const int jj = warp;
#pragma unroll
		for (int f = 0; f < 4; f++) {
			const int nbv = sNb[e * 4 + f];
			const long long le = nbv - e0;
			if (nbv < 0 || le < 0 || le >= nloc) {
				const T *g = nbv >= 0 ? p.w_in + (long long)nbv * 60 + ((sPm[e * 4 + f] >> (4 * jj)) & 15) * 6
									  : p.btrace + ((long long)(-nbv - 1) * 6 + jj) * 6;
#pragma unroll
				for (int c = 0; c < 6; c++)
					pre[f][c] = __ldg(g + c);
			} else {
#pragma unroll
				for (int c = 0; c < 6; c++)
					pre[f][c] = T(0);
			}
		}
	}

	// ---- C: reference derivatives of field `warp`, two physical directions ----
	const int c = warp; // field
	const int a = c % 3;
	if (live) {
		T w[10];
#pragma unroll
		for (int j = 0; j < 10; j++)
			w[j] = sW[(j * 6 + c) * P + e];
		T cod[3][3];
#pragma unroll
		for (int r = 0; r < 3; r++)
#pragma unroll
			for (int q = 0; q < 3; q++)
				cod[r][q] = sG[(3 * r + q) * P + e];
		const int d1 = (a + 1) % 3, d2 = (a + 2) % 3;
		T cd1[3], cd2[3];
#pragma unroll
		for (int k = 0; k < 3; k++) {
			cd1[k] = d1 == 0 ? cod[0][k] : (d1 == 1 ? cod[1][k] : cod[2][k]);
			cd2[k] = d2 == 0 ? cod[0][k] : (d2 == 1 ? cod[1][k] : cod[2][k]);
		}
		T r[3][10];
		ref_derivatives<T, SPARSE>(tb, w, r);
#pragma unroll
		for (int i = 0; i < 10; i++) {
			sX[((c * 2 + 0) * 10 + i) * P + e] = cd1[0] * r[0][i] + cd1[1] * r[1][i] + cd1[2] * r[2][i];
			sX[((c * 2 + 1) * 10 + i) * P + e] = cd2[0] * r[0][i] + cd2[1] * r[1][i] + cd2[2] * r[2][i];
		}
	}

	// ---- B: upwind flux; warp w takes face node jj = w of the 4 faces ----
	if (live) {
		const int jj = warp;
		T cod[3][3];
#pragma unroll
		for (int r = 0; r < 3; r++)
#pragma unroll
			for (int q = 0; q < 3; q++)
				cod[r][q] = sG[(3 * r + q) * P + e];
#pragma unroll
		for (int f = 0; f < 4; f++) {
			const int s = 6 * f + jj;
			const int qo = tb.f2n[f][jj]; // warp-uniform: constant-cache broadcast
			T wL[6], wR[6], vn[3], F[6];
#pragma unroll
			for (int c = 0; c < 6; c++)
				wL[c] = sW[(qo * 6 + c) * P + e];
			const int nbv = sNb[e * 4 + f];
			const long long le = nbv - e0;
			if (nbv >= 0 && le >= 0 && le < nloc) {
				const int qn = (sPm[e * 4 + f] >> (4 * jj)) & 15;
#pragma unroll
				for (int c = 0; c < 6; c++)
					wR[c] = sW[(qn * 6 + c) * P + (int)le];
			} else {
#pragma unroll
				for (int c = 0; c < 6; c++)
					wR[c] = pre[f][c];
			}
			// own scaled outward normal codtau . n_ref(f): the reference
			// normals are -e_0, -e_1, -e_2 and (1,1,1)/sqrt(3), face 3 scaled by
			// sqrt(3) (simulation.c:377-395; checked at attach)
#pragma unroll
			for (int a2 = 0; a2 < 3; a2++)
				vn[a2] = f < 3 ? -cod[a2][f] : (cod[a2][0] + cod[a2][1] + cod[a2][2]) * tb.n3scale;
			upwind_flux<T>(wL, wR, vn, F);
#pragma unroll
			for (int c = 0; c < 6; c++)
				sF[(s * 6 + c) * P + e] = F[c];
		}
	}

	__syncthreads();

	// ---- D: residual of field c, lift, RK update ----
	if (live) {
		// R_E,b = dH_{b+2}/dx_{b+1} - dH_{b+1}/dx_{b+2};  R_H,b = -(same with E)
		const int X = c / 3, b = a;
		const int fa = 3 * (1 - X) + (b + 2) % 3; // field whose "d2" slot holds d_{b+1}
		const int fb = 3 * (1 - X) + (b + 1) % 3; // field whose "d1" slot holds d_{b+2}
		const T sgn = X == 0 ? T(1) : T(-1);
		T R[10];
#pragma unroll
		for (int i = 0; i < 10; i++)
			R[i] = sgn * (sX[((fa * 2 + 1) * 10 + i) * P + e] - sX[((fb * 2 + 0) * 10 + i) * P + e]);
#pragma unroll
		for (int f = 0; f < 4; f++) {
			T Fc[6];
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				Fc[jj] = sF[((f * 6 + jj) * 6 + c) * P + e];
#pragma unroll
			for (int ii = 0; ii < 6; ii++) {
				T acc = T(0);
#pragma unroll
				for (int jj = 0; jj < 6; jj++)
					if (!SPARSE || (smask(ii) >> jj & 1))
						acc += tb.S[ii][jj] * Fc[jj];
				R[f2n(f, ii)] += acc;
			}
		}
		const T inv_det = T(1) / sG[9 * P + e];
		const T A = (T)p.A, B = (T)p.B;
		const T dt = p.einst ? (T)p.dt_tab[p.einst[e0 + e]] : (T)p.dt;
		T dwv[10];
		lift_minv<T>(tb, R, dwv);
#pragma unroll
		for (int i = 0; i < 10; i++) {
			const T dw = dwv[i];
			const int o = (i * 6 + c) * P + e;
			const T k2 = (p.stage0 ? T(0) : A * sK[o]) - dt * (dw * inv_det);
			sK[o] = k2;
			sW[o] = sW[o] + B * k2;
		}
	}
	__syncthreads();

	// ---- E: write the tile back ----
	{
		constexpr int VPC = 16 / sizeof(T);
		const int nch = nloc * 60 / VPC;
		uint4 *gw = reinterpret_cast<uint4 *>(p.w_out + e0 * 60);
		uint4 *gk = reinterpret_cast<uint4 *>(p.k2 + e0 * 60);
		for (int ch = tid; ch < nch; ch += kRk3Threads) {
			const int v0 = ch * VPC;
			const int ee = v0 / 60, k = v0 % 60;
			uint4 av, bv;
			T *ap = reinterpret_cast<T *>(&av);
			T *bp = reinterpret_cast<T *>(&bv);
#pragma unroll
			for (int q = 0; q < VPC; q++) {
				ap[q] = sW[(k + q) * P + ee];
				bp[q] = sK[(k + q) * P + ee];
			}
			__stcs(gw + ch, av);
			if (p.write_k2)
				__stcs(gk + ch, bv);
		}
	}
}

// P2 structural-zero pattern check for the tables handed to attach.
bool rk3_tables_sparse(const gdn_cuda_tables *t)
{
	for (int k = 0; k < 3; k++)
		for (int i = 0; i < 10; i++)
			for (int j = 0; j < 10; j++)
				if (!(dmask(k, i) >> j & 1) && !(t->internal[i][j][k] < 1e-15 && t->internal[i][j][k] > -1e-15))
					return false;
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++)
			if (!(smask(i) >> j & 1) && t->face_scal[i][j] != 0.0)
				return false;
	return true;
}

bool rk3_tables_standard_faces(const gdn_cuda_tables *t)
{
	for (int f = 0; f < 4; f++)
		for (int j = 0; j < 6; j++)
			if (t->face2node[f][j] != f2n(f, j))
				return false;
	// reference normals -e_0, -e_1, -e_2, (1, 1, 1)/sqrt(3)
	for (int f = 0; f < 3; f++)
		for (int k = 0; k < 3; k++)
			if (t->ref_normal[f][k] != (k == f ? -1.0 : 0.0))
				return false;
	for (int k = 0; k < 3; k++)
		if (!(std::fabs(t->ref_normal[3][k] - 0.57735026918962576) < 1e-15))
			return false;
	return true;
}

template <typename T>
int prepare_rk3()
{
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  Rk3Smem<T>::bytes));
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  Rk3Smem<T>::bytes));
	return GDN_CUDA_OK;
}

template <typename T>
int launch_rk3_stage(const Rk3Params<T> &p, cudaStream_t s)
{
	const long long nblk = (p.ne + kRk3Tile - 1) / kRk3Tile;
	if (p.sparse)
		rk3_stage_kernel<T, true><<<(unsigned)nblk, kRk3Threads, Rk3Smem<T>::bytes, s>>>(p);
	else
		rk3_stage_kernel<T, false><<<(unsigned)nblk, kRk3Threads, Rk3Smem<T>::bytes, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template int prepare_rk3<double>();
template int prepare_rk3<float>();
template int launch_rk3_stage<double>(const Rk3Params<double> &, cudaStream_t);
template int launch_rk3_stage<float>(const Rk3Params<float> &, cudaStream_t);

} // namespace gdn
