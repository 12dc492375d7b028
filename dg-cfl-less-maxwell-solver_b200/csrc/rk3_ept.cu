// HP-1, element-per-thread variant of the RK3 stage kernel.
//
// Same arithmetic as rk3_stage_kernel (rk3.cu): R = (curl H, -curl E) +
// sum_faces S F_upwind, dw = Minv R / det, low-storage RK update.  Here one
// thread owns one element for the whole stage and keeps its 60 residual
// accumulators in registers; shared memory is used only to turn the
// element-major global layout into coalesced 16-byte transfers (padded
// [value][element] tiles) and as the source of in-tile neighbour traces.  No
// value is exchanged between threads except through those tiles, so the
// instruction count per element is close to the arithmetic itself.
#include "common.cuh"
#include "kernels.h"

namespace gdn {

constexpr int kEptTile = 128; // elements (= threads) per CTA

template <typename T>
struct EptSmem {
	static constexpr int P = kEptTile + 1;
	static constexpr int bytes = (60 + 60 + 10) * P * (int)sizeof(T);
};

template <typename T, bool SPARSE>
__global__ void __launch_bounds__(kEptTile) rk3_stage_ept_kernel(Rk3Params<T> p)
{
	constexpr int TE = kEptTile, P = EptSmem<T>::P;
	constexpr int VPC = 16 / sizeof(T);
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T *sW = reinterpret_cast<T *>(smem_raw); // [60][P]
	T *sK = sW + 60 * P; // [60][P]
	T *sG = sK + 60 * P; // [10][P]
	const Tables<T> &tb = tab<T>();
	const int tid = threadIdx.x;
	const long long e0 = (long long)blockIdx.x * TE;
	const int nloc = (int)min((long long)TE, p.ne - e0);
	const int nch = nloc * 60 / VPC;

	// ---- stage the tile: 16-byte loads, transposed stores ----
	{
		const uint4 *gw = reinterpret_cast<const uint4 *>(p.w_in + e0 * 60);
		const uint4 *gk = reinterpret_cast<const uint4 *>(p.k2 + e0 * 60);
		for (int ch = tid; ch < nch; ch += TE) {
			const int v0 = ch * VPC;
			const int e = v0 / 60, k = v0 % 60;
			const uint4 a = __ldg(gw + ch);
			const T *av = reinterpret_cast<const T *>(&a);
			if (!p.stage0) {
				const uint4 b = __ldcs(gk + ch);
				const T *bv = reinterpret_cast<const T *>(&b);
#pragma unroll
				for (int q = 0; q < VPC; q++)
					sK[(k + q) * P + e] = bv[q];
			}
#pragma unroll
			for (int q = 0; q < VPC; q++)
				sW[(k + q) * P + e] = av[q];
		}
		for (int v = tid; v < nloc * 10; v += TE)
			sG[(v % 10) * P + v / 10] = p.geom[e0 * 10 + v];
	}
	const int e = tid;
	const bool live = e < nloc;
	int4 nb4 = make_int4(0, 0, 0, 0), pm4 = make_int4(0, 0, 0, 0);
	if (live) {
		nb4 = __ldg(reinterpret_cast<const int4 *>(p.nb) + e0 + e);
		pm4 = __ldg(reinterpret_cast<const int4 *>(p.perm) + e0 + e);
	}
	__syncthreads();

	T R[60];
#pragma unroll
	for (int k = 0; k < 60; k++)
		R[k] = T(0);
	T cod[3][3];
	T det = T(1);
	if (live) {
#pragma unroll
		for (int r = 0; r < 3; r++)
#pragma unroll
			for (int q = 0; q < 3; q++)
				cod[r][q] = sG[(3 * r + q) * P + e];
		det = sG[9 * P + e];

		// ---- volume: field by field, the two physical derivatives the curl
		// needs, scattered into R ----
#pragma unroll
		for (int c = 0; c < 6; c++) {
			const int a = c % 3, X = c / 3;
			const int d1 = (a + 1) % 3, d2 = (a + 2) % 3;
			T w[10];
#pragma unroll
			for (int j = 0; j < 10; j++)
				w[j] = sW[(j * 6 + c) * P + e];
#pragma unroll
			for (int i = 0; i < 10; i++) {
				T r[3];
#pragma unroll
				for (int k = 0; k < 3; k++) {
					T acc = T(0);
#pragma unroll
					for (int j = 0; j < 10; j++)
						if (!SPARSE || (dmask(k, i) >> j & 1))
							acc += tb.D[k][i][j] * w[j];
					r[k] = acc;
				}
				const T g1 = cod[d1][0] * r[0] + cod[d1][1] * r[1] + cod[d1][2] * r[2]; // d_{a+1} X_a
				const T g2 = cod[d2][0] * r[0] + cod[d2][1] * r[1] + cod[d2][2] * r[2]; // d_{a+2} X_a
				// curl_b X = d_{b+1} X_{b+2} - d_{b+2} X_{b+1}: g1 enters curl_{a-1}
				// with -, g2 enters curl_{a+1} with +; R_E = curl H, R_H = -curl E
				const int om = 3 * (1 - X); // output block
				const T s = X == 1 ? T(1) : T(-1);
				R[i * 6 + om + (a + 2) % 3] -= s * g1;
				R[i * 6 + om + (a + 1) % 3] += s * g2;
			}
		}

		// ---- faces: upwind flux at the 6 nodes of each face, lifted by S ----
		const int nbs[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
		const int pms[4] = {pm4.x, pm4.y, pm4.z, pm4.w};
#pragma unroll
		for (int f = 0; f < 4; f++) {
			T vn[3];
#pragma unroll
			for (int a2 = 0; a2 < 3; a2++)
				vn[a2] = f < 3 ? -cod[a2][f] : (cod[a2][0] + cod[a2][1] + cod[a2][2]) * tb.n3scale;
			const int nbv = nbs[f];
			const long long le = nbv - e0;
			const bool intile = nbv >= 0 && le >= 0 && le < nloc;
#pragma unroll
			for (int jj = 0; jj < 6; jj++) {
				const int qo = f2n(f, jj);
				T wL[6], wR[6], F[6];
#pragma unroll
				for (int c = 0; c < 6; c++)
					wL[c] = sW[(qo * 6 + c) * P + e];
				if (intile) {
					const int qn = (pms[f] >> (4 * jj)) & 15;
#pragma unroll
					for (int c = 0; c < 6; c++)
						wR[c] = sW[(qn * 6 + c) * P + (int)le];
				} else {
					// out-of-tile neighbour, or boundary data at the stage time
					const T *g = nbv >= 0 ? p.w_in + (long long)nbv * 60 + ((pms[f] >> (4 * jj)) & 15) * 6
										  : p.btrace + ((long long)(-nbv - 1) * 6 + jj) * 6;
#pragma unroll
					for (int c = 0; c < 6; c++)
						wR[c] = __ldg(g + c);
				}
				upwind_flux<T>(wL, wR, vn, F);
				// column jj of S: R[node(ii)] += S[ii][jj] F
#pragma unroll
				for (int ii = 0; ii < 6; ii++)
					if (!SPARSE || (smask(ii) >> jj & 1)) {
						const T sij = tb.S[ii][jj];
#pragma unroll
						for (int c = 0; c < 6; c++)
							R[f2n(f, ii) * 6 + c] += sij * F[c];
					}
			}
		}
	}
	// every thread has read its neighbours' old values: the tile may now be
	// overwritten with the new state
	__syncthreads();
	if (live) {
		const T inv_det = T(1) / det;
		const T A = (T)p.A, B = (T)p.B;
		const T dt = p.einst ? (T)p.dt_tab[p.einst[e0 + e]] : (T)p.dt;
#pragma unroll
		for (int c = 0; c < 6; c++) {
#pragma unroll
			for (int i = 0; i < 10; i++) {
				T dw = T(0);
#pragma unroll
				for (int j = 0; j < 10; j++)
					dw += tb.Minv[i][j] * R[j * 6 + c];
				const int o = (i * 6 + c) * P + e;
				const T k2 = (p.stage0 ? T(0) : A * sK[o]) - dt * (dw * inv_det);
				sK[o] = k2;
				sW[o] = sW[o] + B * k2;
			}
		}
	}
	__syncthreads();
	{
		uint4 *gw = reinterpret_cast<uint4 *>(p.w_out + e0 * 60);
		uint4 *gk = reinterpret_cast<uint4 *>(p.k2 + e0 * 60);
		for (int ch = tid; ch < nch; ch += TE) {
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

template <typename T>
int prepare_rk3_ept()
{
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_ept_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  EptSmem<T>::bytes));
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_ept_kernel<T, false>,
									  cudaFuncAttributeMaxDynamicSharedMemorySize, EptSmem<T>::bytes));
	return GDN_CUDA_OK;
}

template <typename T>
int launch_rk3_stage_ept(const Rk3Params<T> &p, cudaStream_t s)
{
	const long long nblk = (p.ne + kEptTile - 1) / kEptTile;
	if (p.sparse)
		rk3_stage_ept_kernel<T, true><<<(unsigned)nblk, kEptTile, EptSmem<T>::bytes, s>>>(p);
	else
		rk3_stage_ept_kernel<T, false><<<(unsigned)nblk, kEptTile, EptSmem<T>::bytes, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template int prepare_rk3_ept<double>();
template int prepare_rk3_ept<float>();
template int launch_rk3_stage_ept<double>(const Rk3Params<double> &, cudaStream_t);
template int launch_rk3_stage_ept<float>(const Rk3Params<float> &, cudaStream_t);

} // namespace gdn
