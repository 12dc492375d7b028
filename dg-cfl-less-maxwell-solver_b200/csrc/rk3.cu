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
// Device layout: the state, k2 and the geometry are stored in tiles of 32
// elements, value-major inside a tile (rk3_tix): value k of element e at
// ((e / 32) * 60 + k) * 32 + e % 32.  A CTA owns one tile with 6 warps, lane =
// element, so every per-element access of a warp is one coalesced 128-byte
// (FP32) row:
//   0  every thread starts the gathers of its 24 neighbour-trace values
//      (face node jj = warp of the 4 faces), asynchronously into its own flux
//      slots in shared memory (cp.async; FP64 with few CTAs per SM: into
//      registers), so that phase 1 hides their latency;
//   1  warp c (field c): the 10 nodal values of field c in registers (kept
//      for the RK update) and the two physical weak derivatives the curl
//      needs, through the P1 basis (p1_weak_derivative: d(phi_i) is linear)
//      with the tables as constant-bank operands; they go to shared memory;
//   2  warp jj: the upwind flux at face node jj of the 4 faces (own traces from
//      the tile) to shared memory;
//   -- the one barrier --
//   3  warp c: R_c = curl part + sum_faces S F_c, lift by Minv, RK update with
//      k2 (loaded before the barrier), coalesced stores.
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

// P2 edge nodes 4..9 and their end vertices (t10.c:37-42 face-node lists)
__host__ __device__ constexpr int edge_end(int e, int side)
{
	constexpr int m[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
	return m[e][side];
}

// Physical weak derivative sum_k g_k . D_k w of a P2 field along one
// direction through the P1 basis: d(phi_i) is linear, so
// int d(phi_i) w_h = (vertex i) g_i (4 u_i - s), (edge p-q) 4 (g_p u_q + g_q u_p)
// with u_l = int lambda_l w_h, s = sum_l u_l and g_l the derivative of
// lambda_l along the direction.  v = 4 u; t = v - s (vertex terms).
template <typename T>
__device__ __forceinline__ void p1_weak_derivative(const T cd[3], const T v[4], const T t[4], T out[10])
{
	const T g[4] = {-(cd[0] + cd[1] + cd[2]), cd[0], cd[1], cd[2]};
#pragma unroll
	for (int i = 0; i < 4; i++)
		out[i] = g[i] * t[i];
#pragma unroll
	for (int e = 0; e < 6; e++) {
		const int a = edge_end(e, 0), b = edge_end(e, 1);
		out[4 + e] = g[a] * v[b] + g[b] * v[a];
	}
}

// Vertex sum, edge sum and, per vertex, the sum over its three edges of a P2
// nodal vector.
template <typename T>
__device__ __forceinline__ void p2_sums(const T x[10], T &sv, T &se, T ev[4])
{
	sv = (x[0] + x[1]) + (x[2] + x[3]);
	se = ((x[4] + x[5]) + (x[6] + x[7])) + (x[8] + x[9]);
#pragma unroll
	for (int l = 0; l < 4; l++) {
		T acc = T(0);
		bool first = true;
#pragma unroll
		for (int e = 0; e < 6; e++)
			if (edge_end(e, 0) == l || edge_end(e, 1) == l) {
				acc = first ? x[4 + e] : acc + x[4 + e];
				first = false;
			}
		ev[l] = acc;
	}
}

// v = Q4 w and t = v - sum(v) / 4 through the symmetry of Q4 (q4_sym: qa on
// two vertices, qb on a vertex and an edge through it, qc on a vertex and an
// edge off it): v_l = (qa sv + qc se) - qa w_l + (qb - qc) ev_l.
template <typename T>
__device__ __forceinline__ void q4_apply_sym(const Tables<T> &tb, const T w[10], T v[4], T t[4])
{
	T sv, se, ev[4];
	p2_sums<T>(w, sv, se, ev);
	const T base = tb.q4_sym[0] * sv + tb.q4_sym[1] * se;
	const T s = tb.q4_sym[4] * sv + tb.q4_sym[5] * se; // sum(v) / 4
#pragma unroll
	for (int l = 0; l < 4; l++) {
		v[l] = base + tb.q4_sym[2] * w[l] + tb.q4_sym[3] * ev[l];
		t[l] = v[l] - s;
	}
}

// dw = Minv R through the symmetry of Minv (minv_sym), 58 operations instead
// of 100: vertex i: m0 sv + m1 se + m3 R_i + m4 ev_i; edge p-q: m1 sv + m2 se
// + m4 (R_p + R_q) + m5 R_e + m6 (ev_p + ev_q).
template <typename T>
__device__ __forceinline__ void lift_minv_sym(const Tables<T> &tb, const T R[10], T dw[10])
{
	T sv, se, ev[4];
	p2_sums<T>(R, sv, se, ev);
	const T bv = tb.minv_sym[0] * sv + tb.minv_sym[1] * se;
	const T be = tb.minv_sym[1] * sv + tb.minv_sym[2] * se;
#pragma unroll
	for (int i = 0; i < 4; i++)
		dw[i] = bv + tb.minv_sym[3] * R[i] + tb.minv_sym[4] * ev[i];
#pragma unroll
	for (int e = 0; e < 6; e++) {
		const int a = edge_end(e, 0), b = edge_end(e, 1);
		dw[4 + e] = be + tb.minv_sym[4] * (R[a] + R[b]) + tb.minv_sym[5] * R[4 + e] + tb.minv_sym[6] * (ev[a] + ev[b]);
	}
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

constexpr int kRk3Threads = 192; // 6 warps, one 32-element tile

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
	return (unsigned)__cvta_generic_to_shared(p);
}
// six values global -> shared, asynchronously: dst[cc * DS] = src[cc * SS]
// for cc < 6.  The strides are compile-time, so the six copies address off
// one shared and one global base register with immediate offsets (separate
// asm statements would each materialise both addresses).
template <typename T, int DS, int SS>
__device__ __forceinline__ void cp_async_6(T *dst, const T *src)
{
	asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n\t"
				 "cp.async.ca.shared.global [%0+%3], [%1+%4], %2;\n\t"
				 "cp.async.ca.shared.global [%0+%5], [%1+%6], %2;\n\t"
				 "cp.async.ca.shared.global [%0+%7], [%1+%8], %2;\n\t"
				 "cp.async.ca.shared.global [%0+%9], [%1+%10], %2;\n\t"
				 "cp.async.ca.shared.global [%0+%11], [%1+%12], %2;" ::"r"(smem_u32(dst)),
				 "l"(src), "n"(sizeof(T)), "n"(1 * DS * (int)sizeof(T)), "n"(1 * SS * (int)sizeof(T)),
				 "n"(2 * DS * (int)sizeof(T)), "n"(2 * SS * (int)sizeof(T)), "n"(3 * DS * (int)sizeof(T)),
				 "n"(3 * SS * (int)sizeof(T)), "n"(4 * DS * (int)sizeof(T)), "n"(4 * SS * (int)sizeof(T)),
				 "n"(5 * DS * (int)sizeof(T)), "n"(5 * SS * (int)sizeof(T))
				 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
	asm volatile("cp.async.wait_all;" ::: "memory");
}
// bring [p, p + bytes) into L2 (16-byte aligned, a multiple of 16 bytes)
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes)
{
	asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <typename T>
struct Rk3Smem {
	static constexpr int P = 33;
	// sX: (field*2 + which)*10 + node, 120 rows (table-product path only);
	// sF: (face*6 + jj)*6 + c, 144 rows
	static constexpr int bytes = (120 + 144) * P * (int)sizeof(T);
	static constexpr int bytes_fact = 144 * P * (int)sizeof(T);
};

// The two autotuned CTA-per-tile variants: register cap (minimum resident
// CTAs per SM) and how the neighbour traces are prefetched (rk3_tile).
template <typename T>
struct Rk3Variants;
template <>
struct Rk3Variants<float> {
	static constexpr int lo = 4, hi = 5;
	static constexpr int pf_lo = 2, pf_hi = 2; // PF_ASYNC: 77 / 64 registers
};
template <>
struct Rk3Variants<double> {
	static constexpr int lo = 2, hi = 3;
	static constexpr int pf_lo = 1, pf_hi = 2; // PF_REG at 2 CTAs per SM, PF_ASYNC at 3
};

// Upwind flux with the halving folded into the face quantities: with
// s = wR + wL, d = wR - wL, n2 = n / 2 and r2 = r / 2 (r = 1 / |n|),
//   F_E = -n2 x s_H + r2 (n (n . d_E) - |n|^2 d_E),  F_H = n2 x s_E + r2 (n (n . d_H) - |n|^2 d_H),
// the flux of upwind_flux (maxwell_num_flux_upwind) up to rounding.
template <typename T>
__device__ __forceinline__ void upwind_flux_h(const T wL[6], const T wR[6], const T n[3], T F[6])
{
	const T nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
	const T r2 = T(0.5) * inv_norm_eps(nn);
	const T h[3] = {T(0.5) * n[0], T(0.5) * n[1], T(0.5) * n[2]};
	T sE[3], sH[3], dE[3], dH[3];
#pragma unroll
	for (int k = 0; k < 3; k++) {
		sE[k] = wR[k] + wL[k];
		sH[k] = wR[3 + k] + wL[3 + k];
		dE[k] = wR[k] - wL[k];
		dH[k] = wR[3 + k] - wL[3 + k];
	}
	const T nE = n[0] * dE[0] + n[1] * dE[1] + n[2] * dE[2];
	const T nH = n[0] * dH[0] + n[1] * dH[1] + n[2] * dH[2];
	F[0] = -(h[1] * sH[2] - h[2] * sH[1]) + r2 * (n[0] * nE - nn * dE[0]);
	F[1] = -(h[2] * sH[0] - h[0] * sH[2]) + r2 * (n[1] * nE - nn * dE[1]);
	F[2] = -(h[0] * sH[1] - h[1] * sH[0]) + r2 * (n[2] * nE - nn * dE[2]);
	F[3] = (h[1] * sE[2] - h[2] * sE[1]) + r2 * (n[0] * nH - nn * dH[0]);
	F[4] = (h[2] * sE[0] - h[0] * sE[2]) + r2 * (n[1] * nH - nn * dH[1]);
	F[5] = (h[0] * sE[1] - h[1] * sE[0]) + r2 * (n[2] * nH - nn * dH[2]);
}

// FP32: the same flux with the (E_k, H_k) component pairs in packed FP32x2
// arithmetic: d = wR - wL and t_k = n_k (n . d) - |n|^2 d_k per pair, the
// cross products from the swapped sums (sH_k, sE_k):
// (F_E, F_H)_k = (1, -1) (h_{k+2} sw_{k+1} - h_{k+1} sw_{k+2}) + r2 t_k.
template <>
__device__ __forceinline__ void upwind_flux_h<float>(const float wL[6], const float wR[6], const float n[3],
													 float F[6])
{
	const float nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
	const float r2 = 0.5f * inv_norm_eps(nn);
	const float2 m1 = make_float2(-1.f, -1.f);
	float2 d[3], sw[3];
#pragma unroll
	for (int k = 0; k < 3; k++) {
		d[k] = __ffma2_rn(make_float2(wL[k], wL[3 + k]), m1, make_float2(wR[k], wR[3 + k]));
		sw[k] = __fadd2_rn(make_float2(wR[3 + k], wR[k]), make_float2(wL[3 + k], wL[k]));
	}
	const float2 nd = __ffma2_rn(make_float2(n[2], n[2]), d[2],
								 __ffma2_rn(make_float2(n[1], n[1]), d[1], __fmul2_rn(make_float2(n[0], n[0]), d[0])));
	const float2 mnn = make_float2(-nn, -nn), rr = make_float2(r2, r2), pm = make_float2(1.f, -1.f);
#pragma unroll
	for (int k = 0; k < 3; k++) {
		const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
		const float h1 = 0.5f * n[k1], h2 = 0.5f * n[k2];
		const float2 t = __ffma2_rn(mnn, d[k], __fmul2_rn(make_float2(n[k], n[k]), nd));
		const float2 u = __ffma2_rn(make_float2(-h1, -h1), sw[k2], __fmul2_rn(make_float2(h2, h2), sw[k1]));
		const float2 Fk = __ffma2_rn(u, pm, __fmul2_rn(rr, t));
		F[k] = Fk.x;
		F[3 + k] = Fk.y;
	}
}

// One tile of 32 elements, phases 1-3 (all threads of the CTA call it: it
// holds the barrier between phases 2 and 3).  Wt[k * 32] is value k of this
// lane's element (global memory or a shared-memory copy of the tile), Gt[q *
// 32] its geometry value q, Kin[k * 32] its k2 value k; nbp / pmp point at its
// neighbour and face-node permutation rows.
// Neighbour-trace prefetch: none (loaded in the flux phase), into registers
// at the start, or copied asynchronously into shared memory at the start.
enum { PF_NONE = 0, PF_REG = 1, PF_ASYNC = 2 };

template <typename T, bool SPARSE, bool FACT, int PF, bool METAL>
__device__ __forceinline__ void rk3_tile(const Rk3Params<T> &p, long long tile, const T *Wt, const T *Gt,
										 const T *Kin, const int4 *nbp, const int4 *pmp, T *sX, T *sF)
{
	constexpr int P = Rk3Smem<T>::P;
	const Tables<T> &tb = tab<T>();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long e = tile * 32 + lane;
	const bool live = e < p.ne;

	int nbk[4] = {0, 0, 0, 0}, pmk[4] = {0, 0, 0, 0};
	T cod[3][3], det = T(1);
	// neighbour traces of this thread's flux slot (face node jj = warp) of face f
	auto load_wR = [&](int f, T out[6]) {
		const int nbv = nbk[f];
		const int jj = warp;
		if (nbv >= 0) {
			const int qn = (pmk[f] >> (4 * jj)) & 15;
			const T *g = p.w_in + rk3_tix(nbv, qn * 6);
#pragma unroll
			for (int c = 0; c < 6; c++)
				out[c] = __ldg(g + c * 32);
		} else {
			const T *g = p.btrace + ((long long)(-nbv - 1) * 6 + jj) * 6;
#pragma unroll
			for (int c = 0; c < 6; c++)
				out[c] = __ldg(g + c);
		}
	};
	// Prefetched at the start so that the volume phase hides their latency:
	// PF_REG into registers, PF_ASYNC into this thread's own flux slots of sF
	// ((f * 6 + jj) * 6 + c, the slots its flux later overwrites).
	T wR[PF == PF_REG ? 4 : 1][6];
	if (live) {
		const int4 nb4 = *nbp;
		const int4 pm4 = *pmp;
		nbk[0] = nb4.x, nbk[1] = nb4.y, nbk[2] = nb4.z, nbk[3] = nb4.w;
		pmk[0] = pm4.x, pmk[1] = pm4.y, pmk[2] = pm4.z, pmk[3] = pm4.w;
		if (PF == PF_REG) {
#pragma unroll
			for (int f = 0; f < 4; f++)
				load_wR(f, wR[PF == PF_REG ? f : 0]);
		}
		if (PF == PF_ASYNC) {
#pragma unroll
			for (int f = 0; f < 4; f++) {
				const int nbv = nbk[f];
				T *d = sF + ((f * 6 + warp) * 6) * P + lane;
				// constant strides in each branch, so the six copies use
				// immediate offsets; 32-bit tile offsets when the state fits
				if (nbv >= 0) {
					const unsigned qn = ((unsigned)pmk[f] >> (4 * warp)) & 15u;
					const T *g = p.idx32 ? p.w_in + (((unsigned)nbv >> 5) * 1920u + qn * 192u + ((unsigned)nbv & 31u))
										 : p.w_in + rk3_tix(nbv, (int)qn * 6);
					cp_async_6<T, P, 32>(d, g);
				} else {
					const T *g = p.btrace + ((long long)(-nbv - 1) * 6 + warp) * 6;
					cp_async_6<T, P, 1>(d, g);
				}
			}
		}
#pragma unroll
		for (int r = 0; r < 3; r++)
#pragma unroll
			for (int q = 0; q < 3; q++)
				cod[r][q] = Gt[(3 * r + q) * 32];
		det = Gt[9 * 32];
	}

	// ---- 1: field c = warp in registers (kept for the RK update); the
	// table-product path also computes its two physical derivatives for the
	// curl into sX (FACT computes the curl's derivatives in phase 3) ----
	const int c = warp;
	const int a = c % 3;
	T w[10];
	if (live) {
#pragma unroll
		for (int j = 0; j < 10; j++)
			w[j] = Wt[(j * 6 + c) * 32];
	}
	if (!FACT && live) {
		const int d1 = (a + 1) % 3, d2 = (a + 2) % 3;
		T cd1[3], cd2[3];
#pragma unroll
		for (int k = 0; k < 3; k++) {
			cd1[k] = d1 == 0 ? cod[0][k] : (d1 == 1 ? cod[1][k] : cod[2][k]);
			cd2[k] = d2 == 0 ? cod[0][k] : (d2 == 1 ? cod[1][k] : cod[2][k]);
		}
		{
			T r[3][10];
			ref_derivatives<T, SPARSE>(tb, w, r);
#pragma unroll
			for (int i = 0; i < 10; i++) {
				sX[((c * 2 + 0) * 10 + i) * P + lane] = cd1[0] * r[0][i] + cd1[1] * r[1][i] + cd1[2] * r[2][i];
				sX[((c * 2 + 1) * 10 + i) * P + lane] = cd2[0] * r[0][i] + cd2[1] * r[1][i] + cd2[2] * r[2][i];
			}
		}
	}

	// ---- 2: upwind flux at face node jj = warp of the 4 faces ----
	if (live) {
		const int jj = warp;
#pragma unroll
		for (int f = 0; f < 4; f++) {
			const int qo = tb.f2n[f][jj]; // warp-uniform: constant-cache broadcast
			T wL[6], vn[3], F[6];
#pragma unroll
			for (int cc = 0; cc < 6; cc++)
				wL[cc] = Wt[(qo * 6 + cc) * 32];
			// own scaled outward normal codtau . n_ref(f): the reference
			// normals are -e_0, -e_1, -e_2 and (1,1,1)/sqrt(3), face 3 scaled by
			// sqrt(3) (simulation.c:377-395; checked at attach)
#pragma unroll
			for (int a2 = 0; a2 < 3; a2++)
				vn[a2] = f < 3 ? -cod[a2][f] : (cod[a2][0] + cod[a2][1] + cod[a2][2]) * tb.n3scale;
			if (PF == PF_ASYNC) {
				if (f == 0)
					cp_async_wait_all();
#pragma unroll
				for (int cc = 0; cc < 6; cc++)
					wR[0][cc] = sF[((f * 6 + jj) * 6 + cc) * P + lane];
			} else if (PF == PF_NONE) {
				load_wR(f, wR[0]);
			}
			if (METAL && nbk[f] < 0) {
				// maxwell_num_flux_boundary_metal (maxwell.c:205-223)
				F[0] = vn[2] * wL[4] - vn[1] * wL[5];
				F[1] = -vn[2] * wL[3] + vn[0] * wL[5];
				F[2] = -vn[0] * wL[4] + vn[1] * wL[3];
				F[3] = F[4] = F[5] = T(0);
			} else {
				upwind_flux_h<T>(wL, wR[PF == PF_REG ? f : 0], vn, F);
			}
#pragma unroll
			for (int cc = 0; cc < 6; cc++)
				sF[((f * 6 + jj) * 6 + cc) * P + lane] = F[cc];
		}
	}
	T k2o[10];
	T *Kt = p.k2 + tile * 60 * 32 + lane;
	if (live && !p.stage0) {
#pragma unroll
		for (int i = 0; i < 10; i++)
			k2o[i] = Kin[(i * 6 + c) * 32];
	}

	__syncthreads();

	// ---- 3: residual of field c, lift, RK update ----
	if (!live)
		return;
	// R_E,b = dH_{b+2}/dx_{b+1} - dH_{b+1}/dx_{b+2};  R_H,b = -(same with E)
	const int X = c / 3, b = a;
	const int fa = 3 * (1 - X) + (b + 2) % 3; // field whose "d2" slot holds d_{b+1}
	const int fb = 3 * (1 - X) + (b + 1) % 3; // field whose "d1" slot holds d_{b+2}
	T R[10];
	if (FACT) {
		// d_{b+1} of field fa and d_{b+2} of field fb through the P1 basis
		// (p1_weak_derivative), their rows read back from the tile (L1)
		T o[2][10];
#pragma unroll
		for (int h = 0; h < 2; h++) {
			const int fld = h ? fb : fa;
			const int d = (b + 1 + h) % 3;
			T wf[10], v[4], t[4], cd[3];
#pragma unroll
			for (int j = 0; j < 10; j++)
				wf[j] = Wt[(j * 6 + fld) * 32];
			q4_apply_sym<T>(tb, wf, v, t);
#pragma unroll
			for (int k = 0; k < 3; k++)
				cd[k] = d == 0 ? cod[0][k] : (d == 1 ? cod[1][k] : cod[2][k]);
			p1_weak_derivative<T>(cd, v, t, o[h]);
		}
#pragma unroll
		for (int i = 0; i < 10; i++)
			R[i] = X == 0 ? o[0][i] - o[1][i] : o[1][i] - o[0][i];
	} else {
		const T sgn = X == 0 ? T(1) : T(-1);
#pragma unroll
		for (int i = 0; i < 10; i++)
			R[i] = sgn * (sX[((fa * 2 + 1) * 10 + i) * P + lane] - sX[((fb * 2 + 0) * 10 + i) * P + lane]);
	}
#pragma unroll
	for (int f = 0; f < 4; f++) {
		T Fc[6];
#pragma unroll
		for (int jj = 0; jj < 6; jj++)
			Fc[jj] = sF[((f * 6 + jj) * 6 + c) * P + lane];
		if (FACT) {
			// S Fc through the triangle's symmetry (s_sym)
			const T bv = tb.s_sym[1] * ((Fc[0] + Fc[1]) + Fc[2]);
			const T be = tb.s_sym[4] * ((Fc[3] + Fc[4]) + Fc[5]);
#pragma unroll
			for (int ii = 0; ii < 3; ii++)
				R[f2n(f, ii)] += bv + tb.s_sym[0] * Fc[ii] + tb.s_sym[2] * Fc[3 + (ii + 1) % 3];
#pragma unroll
			for (int k = 0; k < 3; k++)
				R[f2n(f, 3 + k)] += be + tb.s_sym[3] * Fc[3 + k] + tb.s_sym[2] * Fc[(k + 2) % 3];
		} else {
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
	}
	const T A = (T)p.A, B = (T)p.B;
	const T dt = p.einst ? (T)p.dt_tab[p.einst[e]] : (T)p.dt;
	const T scale = dt / det;
	T dwv[10];
	if (FACT)
		lift_minv_sym<T>(tb, R, dwv);
	else
		lift_minv<T>(tb, R, dwv);
	T *Wo = p.w_out + tile * 60 * 32 + lane;
#pragma unroll
	for (int i = 0; i < 10; i++) {
		const T k2 = p.stage0 ? -(scale * dwv[i]) : A * k2o[i] - scale * dwv[i];
		Wo[(i * 6 + c) * 32] = w[i] + B * k2;
		if (p.write_k2)
			Kt[(i * 6 + c) * 32] = k2;
	}
}

// One CTA per tile, everything read from global memory.
// MINB resident CTAs per SM: ptxas derives the register cap, including the
// split of the register file between the SM's four schedulers (18 warps of 3
// CTAs leave 5 warps on one scheduler: 96 registers, not 65536 / 576)
template <typename T, bool SPARSE, bool FACT, int MINB, int PF, bool METAL>
__global__ void __launch_bounds__(kRk3Threads, MINB) rk3_stage_kernel(Rk3Params<T> p)
{
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T *sX = reinterpret_cast<T *>(smem_raw); // [120][P]
	T *sF = FACT ? sX : sX + 120 * Rk3Smem<T>::P; // [144][P] (FACT: no sX)
	const long long tile = blockIdx.x;
	const int lane = threadIdx.x & 31;
	const long long e = tile * 32 + lane;
	const long long ec = e < p.ne ? e : p.ne - 1;
	// the tile that starts on this SM about one CTA lifetime from now (l2_ahead
	// = resident CTAs on the GPU): its state, k2, geometry and neighbour rows
	// into L2, so that its first loads are L2 hits
	if (threadIdx.x == 0 && p.l2_ahead > 0) {
		const long long tn = tile + p.l2_ahead;
		const long long nt = (p.ne + 31) / 32;
		if (tn < nt) {
			const unsigned wb = 60 * 32 * sizeof(T);
			prefetch_l2(p.w_in + tn * 60 * 32, wb);
			if (!p.stage0)
				prefetch_l2(p.k2 + tn * 60 * 32, wb);
			prefetch_l2(p.geom + tn * 10 * 32, 10 * 32 * sizeof(T));
			const unsigned nbb = (unsigned)((p.ne - tn * 32 < 32 ? p.ne - tn * 32 : 32) * 16);
			prefetch_l2(p.nb + tn * 32 * 4, nbb);
			prefetch_l2(p.perm + tn * 32 * 4, nbb);
		}
	}
	const T *Wt = p.w_in + tile * 60 * 32 + lane;
	rk3_tile<T, SPARSE, FACT, PF, METAL>(p, tile, Wt, p.geom + tile * 10 * 32 + lane, p.k2 + tile * 60 * 32 + lane,
										 reinterpret_cast<const int4 *>(p.nb) + ec,
										 reinterpret_cast<const int4 *>(p.perm) + ec, sX, sF);
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

// Q4[l][j] = 4 int lambda_l phi_j = 4 sum_m lambda_l(x_m) M[m][j] (lambda_l is
// linear, so its P2 interpolant is exact); the vertex diagonal is zero for
// the P2 basis and is set to zero (rk3_tables_factor checks the whole
// product).
void rk3_q4(const gdn_cuda_tables *t, double q4[4][10])
{
	for (int l = 0; l < 4; l++)
		for (int j = 0; j < 10; j++) {
			double acc = t->mass[l][j];
			for (int e = 0; e < 6; e++)
				if (edge_end(e, 0) == l || edge_end(e, 1) == l)
					acc += 0.5 * t->mass[4 + e][j];
			q4[l][j] = j == l ? 0.0 : 4.0 * acc;
		}
}

// How nodes i and j of the P2 tetrahedron sit relative to each other: 0 same
// vertex, 1 two vertices, 2 vertex on the edge, 3 vertex off the edge, 4 same
// edge, 5 edges sharing a vertex, 6 opposite edges.
static int node_pair_kind(int i, int j)
{
	if (i < 4 && j < 4)
		return i == j ? 0 : 1;
	if (i < 4 || j < 4) {
		const int v = i < 4 ? i : j, e = (i < 4 ? j : i) - 4;
		return (edge_end(e, 0) == v || edge_end(e, 1) == v) ? 2 : 3;
	}
	if (i == j)
		return 4;
	const int a0 = edge_end(i - 4, 0), a1 = edge_end(i - 4, 1), b0 = edge_end(j - 4, 0), b1 = edge_end(j - 4, 1);
	return (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) ? 5 : 6;
}

// Coefficients of q4_apply_sym and lift_minv_sym from one representative
// entry per kind (rk3_tables_factor checks that every entry equals its kind's).
void rk3_sym_coeffs(const gdn_cuda_tables *t, double q4_sym[6], double minv_sym[7], double s_sym[5])
{
	const double(*S)[6] = t->face_scal; // face nodes: vertices 0-2, edges 01, 12, 20
	s_sym[0] = S[0][0] - S[0][1];
	s_sym[1] = S[0][1];
	s_sym[2] = S[0][4]; // vertex 0 and its opposite edge 12
	s_sym[3] = S[3][3] - S[3][4];
	s_sym[4] = S[3][4];
	double q4[4][10];
	rk3_q4(t, q4);
	const double qa = q4[0][1], qb = q4[0][4], qc = q4[0][5]; // edge 4 = 0-1, edge 5 = 1-2
	q4_sym[0] = qa;
	q4_sym[1] = qc;
	q4_sym[2] = -qa;
	q4_sym[3] = qb - qc;
	q4_sym[4] = 0.75 * qa; // sum_l v_l = 3 qa sv + 2 (qb + qc) se
	q4_sym[5] = 0.5 * (qb + qc);
	const double(*M)[10] = t->inv_mass;
	const double vv0 = M[0][0], vv1 = M[0][1], vin = M[0][4], vout = M[0][5];
	const double ee0 = M[4][4], ee1 = M[4][5], ee2 = M[4][9]; // edges 0-1 / 1-2 / 2-3
	minv_sym[0] = vv1;
	minv_sym[1] = vout;
	minv_sym[2] = ee2;
	minv_sym[3] = vv0 - vv1;
	minv_sym[4] = vin - vout;
	minv_sym[5] = ee0 - 2.0 * ee1 + ee2;
	minv_sym[6] = ee1 - ee2;
}

// The symmetric forms: every entry of Q4 and Minv equals its kind's
// representative (to 1e-15 of the largest entry).
static bool rk3_tables_symmetric(const gdn_cuda_tables *t)
{
	double q4[4][10], qmax = 0.0, mmax = 0.0;
	rk3_q4(t, q4);
	for (int l = 0; l < 4; l++)
		for (int j = 0; j < 10; j++)
			qmax = std::fmax(qmax, std::fabs(q4[l][j]));
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++)
			mmax = std::fmax(mmax, std::fabs(t->inv_mass[i][j]));
	const double qrep[4] = {0.0, q4[0][1], q4[0][4], q4[0][5]};
	for (int l = 0; l < 4; l++)
		for (int j = 0; j < 10; j++)
			if (!(std::fabs(q4[l][j] - qrep[node_pair_kind(l, j)]) <= 1e-15 * qmax))
				return false;
	const double(*M)[10] = t->inv_mass;
	const double mrep[7] = {M[0][0], M[0][1], M[0][4], M[0][5], M[4][4], M[4][5], M[4][9]};
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++)
			if (!(std::fabs(M[i][j] - mrep[node_pair_kind(i, j)]) <= 1e-15 * mmax))
				return false;
	// face mass: kinds on the P2 triangle (face-local vertex i is opposite the
	// edge 3 + (i + 1) % 3); a vertex and an edge through it: structural zero
	const double(*S)[6] = t->face_scal;
	double smax = 0.0;
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++)
			smax = std::fmax(smax, std::fabs(S[i][j]));
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++) {
			double rep;
			if (i < 3 && j < 3)
				rep = i == j ? S[0][0] : S[0][1];
			else if (i >= 3 && j >= 3)
				rep = i == j ? S[3][3] : S[3][4];
			else {
				const int v = i < 3 ? i : j, ed = i < 3 ? j : i;
				rep = ed == 3 + (v + 1) % 3 ? S[0][4] : 0.0;
			}
			if (!(std::fabs(S[i][j] - rep) <= 1e-15 * smax))
				return false;
		}
	return true;
}

// D_k[i][j] = sum_l G_k[i][l] Q4[l][j] / 4 with G_k the P1 coefficients of
// d_k(phi_i) (reference vertices 0, e_0, e_1, e_2), to 1e-15; and Q4 and Minv
// have the tetrahedral symmetry the factored kernel uses.
bool rk3_tables_factor(const gdn_cuda_tables *t)
{
	if (!rk3_tables_symmetric(t))
		return false;
	double q4[4][10];
	rk3_q4(t, q4);
	for (int k = 0; k < 3; k++) {
		double dl[4] = {-1.0, 0.0, 0.0, 0.0}; // d_k lambda_l
		dl[k + 1] = 1.0;
		for (int i = 0; i < 10; i++) {
			double G[4] = {0.0, 0.0, 0.0, 0.0};
			if (i < 4) {
				for (int l = 0; l < 4; l++)
					G[l] = dl[i] * (l == i ? 3.0 : -1.0);
			} else {
				const int a = edge_end(i - 4, 0), b = edge_end(i - 4, 1);
				G[a] += 4.0 * dl[b];
				G[b] += 4.0 * dl[a];
			}
			for (int j = 0; j < 10; j++) {
				double d = 0.0;
				for (int l = 0; l < 4; l++)
					d += G[l] * 0.25 * q4[l][j];
				if (!(std::fabs(d - t->internal[i][j][k]) <= 1e-15))
					return false;
			}
		}
	}
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

#define GDN_RK3_TRY(expr)                                                                                         \
	do {                                                                                                           \
		int _rc = (expr);                                                                                          \
		if (_rc != GDN_CUDA_OK)                                                                                    \
			return _rc;                                                                                            \
	} while (0)

template <typename T, bool FA>
constexpr int rk3_smem_bytes()
{
	return FA ? Rk3Smem<T>::bytes_fact : Rk3Smem<T>::bytes;
}

template <typename T, bool SP, bool FA, bool METAL>
static int prepare_rk3_one()
{
	typedef Rk3Variants<T> V;
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_kernel<T, SP, FA, V::lo, V::pf_lo, METAL>,
									  cudaFuncAttributeMaxDynamicSharedMemorySize, rk3_smem_bytes<T, FA>()));
	GDN_CUDA_TRY(cudaFuncSetAttribute(rk3_stage_kernel<T, SP, FA, V::hi, V::pf_hi, METAL>,
									  cudaFuncAttributeMaxDynamicSharedMemorySize, rk3_smem_bytes<T, FA>()));
	return GDN_CUDA_OK;
}

template <typename T>
int prepare_rk3()
{
	GDN_RK3_TRY((prepare_rk3_one<T, true, true, false>()));
	GDN_RK3_TRY((prepare_rk3_one<T, true, false, false>()));
	GDN_RK3_TRY((prepare_rk3_one<T, false, false, false>()));
	GDN_RK3_TRY((prepare_rk3_one<T, true, true, true>()));
	GDN_RK3_TRY((prepare_rk3_one<T, true, false, true>()));
	GDN_RK3_TRY((prepare_rk3_one<T, false, false, true>()));
	return GDN_CUDA_OK;
}

template <typename T, bool SP, bool FA, bool METAL>
static void launch_rk3_one(const Rk3Params<T> &pin, int variant, cudaStream_t s)
{
	typedef Rk3Variants<T> V;
	Rk3Params<T> p = pin;
	// L2 prefetch distance: the CTAs resident on the GPU at this variant's cap
	// (FP32), half of them (FP64).  96^3 ms per step, FP32 / FP64, for none,
	// half, one and two times the resident CTAs: 4.35 / 9.45, 4.25 / 9.03,
	// 4.24 / 9.14, 4.32 / 9.67.
	const int resident = p.num_sms * (variant == 0 ? V::lo : V::hi);
	p.l2_ahead = p.l2_ahead ? (sizeof(T) == 8 ? resident / 2 : resident) : 0;
	const unsigned nblk = (unsigned)((p.ne + 31) / 32);
	const int sm = rk3_smem_bytes<T, FA>();
	if (variant == 0)
		rk3_stage_kernel<T, SP, FA, V::lo, V::pf_lo, METAL><<<nblk, kRk3Threads, sm, s>>>(p);
	else
		rk3_stage_kernel<T, SP, FA, V::hi, V::pf_hi, METAL><<<nblk, kRk3Threads, sm, s>>>(p);
}

template <typename T, bool METAL>
static void launch_rk3_tables(const Rk3Params<T> &p, int variant, cudaStream_t s)
{
	if (p.sparse && p.fact)
		launch_rk3_one<T, true, true, METAL>(p, variant, s);
	else if (p.sparse)
		launch_rk3_one<T, true, false, METAL>(p, variant, s);
	else
		launch_rk3_one<T, false, false, METAL>(p, variant, s);
}

// variant 0: register cap for Rk3Variants::lo CTAs per SM, 1: for ::hi
template <typename T>
int launch_rk3_stage(const Rk3Params<T> &p, int variant, cudaStream_t s)
{
	if (p.bc_metal)
		launch_rk3_tables<T, true>(p, variant, s);
	else
		launch_rk3_tables<T, false>(p, variant, s);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

int rk3_min_blocks(int precision_fp64, int variant)
{
	if (precision_fp64)
		return variant == 0 ? Rk3Variants<double>::lo : Rk3Variants<double>::hi;
	return variant == 0 ? Rk3Variants<float>::lo : Rk3Variants<float>::hi;
}

// reference layout [e][node i][field c] (FP64, local elements 0..ne-1) <->
// tiles (global elements e0 + e)
template <typename T>
__global__ void rk3_to_tiles_kernel(const double *__restrict__ src, T *__restrict__ dst, long long e0, long long ne)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= ne * 60)
		return;
	const long long e = u / 60;
	const int k = (int)(u % 60);
	dst[rk3_tix(e0 + e, k)] = (T)src[u];
}
template <typename T>
__global__ void rk3_from_tiles_kernel(const T *__restrict__ src, double *__restrict__ dst, long long e0, long long ne)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= ne * 60)
		return;
	const long long e = u / 60;
	const int k = (int)(u % 60);
	dst[u] = (double)src[rk3_tix(e0 + e, k)];
}
// geometry [e][10] FP64 -> tiles of T
template <typename T>
__global__ void geom_to_tiles_kernel(const double *__restrict__ g, T *__restrict__ out, long long ne)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= ne * 10)
		return;
	const long long e = u / 10;
	const int q = (int)(u % 10);
	out[((e >> 5) * 10 + q) * 32 + (e & 31)] = (T)g[u];
}

template <typename T>
int launch_rk3_to_tiles(const double *src, T *dst, long long e0, long long ne, cudaStream_t s)
{
	if (ne <= 0)
		return GDN_CUDA_OK;
	rk3_to_tiles_kernel<T><<<(unsigned)((ne * 60 + 255) / 256), 256, 0, s>>>(src, dst, e0, ne);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template <typename T>
int launch_rk3_from_tiles(const T *src, double *dst, long long e0, long long ne, cudaStream_t s)
{
	if (ne <= 0)
		return GDN_CUDA_OK;
	rk3_from_tiles_kernel<T><<<(unsigned)((ne * 60 + 255) / 256), 256, 0, s>>>(src, dst, e0, ne);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template <typename T>
int launch_geom_to_tiles(const double *g, T *out, long long ne, cudaStream_t s)
{
	geom_to_tiles_kernel<T><<<(unsigned)((ne * 10 + 255) / 256), 256, 0, s>>>(g, out, ne);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template int prepare_rk3<double>();
template int prepare_rk3<float>();
template int launch_rk3_stage<double>(const Rk3Params<double> &, int, cudaStream_t);
template int launch_rk3_stage<float>(const Rk3Params<float> &, int, cudaStream_t);
template int launch_rk3_to_tiles<double>(const double *, double *, long long, long long, cudaStream_t);
template int launch_rk3_to_tiles<float>(const double *, float *, long long, long long, cudaStream_t);
template int launch_rk3_from_tiles<double>(const double *, double *, long long, long long, cudaStream_t);
template int launch_rk3_from_tiles<float>(const float *, double *, long long, long long, cudaStream_t);
template int launch_geom_to_tiles<double>(const double *, double *, long long, cudaStream_t);
template int launch_geom_to_tiles<float>(const double *, float *, long long, cudaStream_t);

} // namespace gdn
