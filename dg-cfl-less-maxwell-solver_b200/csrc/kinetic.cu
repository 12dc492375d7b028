// HP-2: the CFL-less kinetic-relaxation step (src/dg/relaxation.c:93-174).
//
// The reference, per step: boundary dofs <- f_eq(w_I(x, t + dt/2));
// for every field iw and velocity iv: sol = M2_iv wn; solve M1_iv sol (KLU);
// swap; relax every dof: f <- omega f_eq(w(f)) + (1 - omega) f.
// With M1 = I + theta dt A and M2 = I - (1 - theta) dt A (relaxation.c:79-83),
// M2 = (1/theta) I - ((1 - theta)/theta) M1, hence
//   M1^-1 M2 f = (1/theta) y - ((1 - theta)/theta) f,   y = M1^-1 f,
// so one block forward substitution per velocity replaces the SpMV + LU
// solve.  M1 is block lower-triangular in a downwind element order (an element
// row couples only to its upwind neighbours, simulation.c:493-604); the host
// builds the level schedule of that order once per velocity and the sweep
// runs level by level, all velocities and all 6 fields of a level in one
// launch.  Per element and velocity the diagonal block is
//   D = I + (theta dt / det) Minv (V + sum_outflow s+ E_f S E_f^T),
//   V_ij = -(v . c_ij), s = v . vn (the L-side scaled normal of each face),
// inverted once at attach in FP64 (G = D^-1); a sweep item computes
//   y_e = G (f_e - (theta dt / det) Minv sum_inflow s- E_f S y_nb|_f).
//
// Sweep order: the state of (element e, velocity v) lives at item index
// k = pos[e * nv + v], its position in the level-sorted item list, so the
// items of one level are contiguous in memory and an item finds everything
// it needs from one record (inflow neighbour items, permutations, v . vn).
#include <climits>

#include <cuda_pipeline_primitives.h>

#include "aux.h"
#include "kernels.h"

namespace gdn {

// own-side v.vn of every element face for every velocity, from the L-side
// normal of each face in the reference's operation order (simulation.c:
// 520-540 + kinetic_num_flux_upwind): the R side gets exactly -s.
__global__ void kin_face_s_kernel(const int *__restrict__ face2elem, long long nf, const double *__restrict__ geom,
								  KinModel km, double *__restrict__ sown64)
{
	const long long F = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (F >= nf)
		return;
	const long long eL = face2elem[4 * F], eR = face2elem[4 * F + 2];
	const int fL = face2elem[4 * F + 1], fR = face2elem[4 * F + 3];
	double cod[3][3], vn[3];
	for (int a = 0; a < 3; a++)
		for (int b = 0; b < 3; b++)
			cod[a][b] = geom[eL * 10 + 3 * a + b];
	gdn_face_normal(cod, c_tab_d.ref_normal, fL, vn);
	for (int v = 0; v < km.nv; v++) {
		const double s = gdn_dot_lr(km.vi + 3 * v, vn);
		sown64[(eL * km.nv + v) * 4 + fL] = s;
		if (eR >= 0)
			sown64[(eR * km.nv + v) * 4 + fR] = -s;
	}
}

// inflow mask: bit f set when element e depends on its neighbour across f
__global__ void kin_mask_kernel(const double *__restrict__ sown64, const int *__restrict__ nb, long long ne, int nv,
								unsigned char *__restrict__ mask)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= ne * nv)
		return;
	const long long e = u / nv;
	unsigned char m = 0;
	for (int f = 0; f < 4; f++)
		if (nb[e * 4 + f] >= 0 && sown64[u * 4 + f] < 0.0)
			m |= (unsigned char)(1 << f);
	mask[u] = m;
}

// G = D^-1 per (element, velocity), FP64 Gauss-Jordan with partial
// pivoting, written at the item's sweep position.
template <typename GT>
__global__ void kin_blocks_kernel(const double *__restrict__ geom, const double *__restrict__ sown64,
								  const int *__restrict__ pos, long long ne, KinModel km, double theta_dt,
								  GT *__restrict__ G, GT *__restrict__ coef, int *__restrict__ bad)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= ne * km.nv)
		return;
	const long long e = u / km.nv;
	const int v = (int)(u % km.nv);
	const Tables<double> &tb = c_tab_d;
	const double *vv = km.vi + 3 * v;
	double cod[3][3];
	for (int a = 0; a < 3; a++)
		for (int b = 0; b < 3; b++)
			cod[a][b] = geom[e * 10 + 3 * a + b];
	const double det = geom[e * 10 + 9];
	// u_k = sum_l v_l codtau[l][k]:  v . c_ij = sum_k u_k int d_k phi_i phi_j
	double uk[3];
	for (int k = 0; k < 3; k++)
		uk[k] = vv[0] * cod[0][k] + vv[1] * cod[1][k] + vv[2] * cod[2][k];
	double F[10][10];
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++)
			F[i][j] = -(uk[0] * tb.D[0][i][j] + uk[1] * tb.D[1][i][j] + uk[2] * tb.D[2][i][j]);
	for (int f = 0; f < 4; f++) {
		const double s = sown64[u * 4 + f];
		const double sp = s > 0.0 ? s : 0.0;
		if (sp == 0.0)
			continue;
		for (int ii = 0; ii < 6; ii++)
			for (int jj = 0; jj < 6; jj++)
				F[tb.f2n[f][ii]][tb.f2n[f][jj]] += sp * tb.S[ii][jj];
	}
	const double c = theta_dt / det;
	double a[10][20];
	for (int i = 0; i < 10; i++) {
		for (int j = 0; j < 10; j++) {
			double acc = 0.0;
			for (int k = 0; k < 10; k++)
				acc += tb.Minv[i][k] * F[k][j];
			a[i][j] = (i == j ? 1.0 : 0.0) + c * acc;
			a[i][10 + j] = i == j ? 1.0 : 0.0;
		}
	}
	for (int k = 0; k < 10; k++) {
		int piv = k;
		for (int r = k + 1; r < 10; r++)
			if (fabs(a[r][k]) > fabs(a[piv][k]))
				piv = r;
		if (piv != k)
			for (int q = 0; q < 20; q++) {
				double t = a[k][q];
				a[k][q] = a[piv][q];
				a[piv][q] = t;
			}
		if (a[k][k] == 0.0) {
			atomicMax(bad, 1);
			return;
		}
		const double inv = 1.0 / a[k][k];
		for (int q = 0; q < 20; q++)
			a[k][q] *= inv;
		for (int r = 0; r < 10; r++)
			if (r != k) {
				const double m = a[r][k];
				if (m != 0.0)
					for (int q = 0; q < 20; q++)
						a[r][q] -= m * a[k][q];
			}
	}
	GT *Gk = G + (long long)pos[u] * 100;
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++)
			Gk[i * 10 + j] = (GT)a[i][10 + j];
	if (v == 0)
		coef[e] = (GT)c;
}

// per-item records of the sweep
template <typename GT>
__global__ void kin_records_kernel(const int *__restrict__ items, const int *__restrict__ pos,
								   const double *__restrict__ sown64, const int *__restrict__ nb,
								   const int *__restrict__ perm, long long nitems, int nv, int4 *__restrict__ rnb,
								   int4 *__restrict__ rpm, GT *__restrict__ rs, int *__restrict__ relem)
{
	const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (k >= nitems)
		return;
	const long long u = items[k];
	const long long e = u / nv;
	const int v = (int)(u % nv);
	int n[4], pm[4];
	for (int f = 0; f < 4; f++) {
		const double s = sown64[u * 4 + f];
		const int nbv = nb[e * 4 + f];
		pm[f] = perm[e * 4 + f];
		rs[k * 4 + f] = (GT)s;
		if (!(s < 0.0))
			n[f] = INT_MIN; // outflow or tangent: no coupling
		else if (nbv >= 0)
			n[f] = pos[(long long)nbv * nv + v];
		else
			n[f] = nbv; // -(boundary face + 1)
	}
	rnb[k] = make_int4(n[0], n[1], n[2], n[3]);
	rpm[k] = make_int4(pm[0], pm[1], pm[2], pm[3]);
	relem[k] = (int)e;
}

template <typename GT>
int launch_kin_setup(const int *face2elem, long long nf, const double *geom, const int *nb, long long ne,
					 const KinModel &km, double *sown64, unsigned char *mask, cudaStream_t s)
{
	kin_face_s_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(face2elem, nf, geom, km, sown64);
	GDN_CUDA_TRY(cudaGetLastError());
	const long long nu = ne * km.nv;
	kin_mask_kernel<<<(unsigned)((nu + 255) / 256), 256, 0, s>>>(sown64, nb, ne, km.nv, mask);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template <typename GT>
int launch_kin_blocks(const double *geom, const double *sown64, const int *items, const int *pos, const int *nb,
					  const int *perm, long long ne, const KinModel &km, double theta_dt, GT *G, GT *coef,
					  int4 *rnb, int4 *rpm, GT *rs, int *relem, int *bad, cudaStream_t s)
{
	const long long nu = ne * km.nv;
	kin_blocks_kernel<GT><<<(unsigned)((nu + 127) / 128), 128, 0, s>>>(geom, sown64, pos, ne, km, theta_dt, G, coef,
																	   bad);
	GDN_CUDA_TRY(cudaGetLastError());
	kin_records_kernel<GT><<<(unsigned)((nu + 255) / 256), 256, 0, s>>>(items, pos, sown64, nb, perm, nu, km.nv, rnb,
																		rpm, rs, relem);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_setup<double>(const int *, long long, const double *, const int *, long long,
									  const KinModel &, double *, unsigned char *, cudaStream_t);
template int launch_kin_blocks<double>(const double *, const double *, const int *, const int *, const int *,
									   const int *, long long, const KinModel &, double, double *, double *, int4 *,
									   int4 *, double *, int *, int *, cudaStream_t);
template int launch_kin_blocks<float>(const double *, const double *, const int *, const int *, const int *,
									  const int *, long long, const KinModel &, double, float *, float *, int4 *,
									  int4 *, float *, int *, int *, cudaStream_t);

// One level of the block forward substitution: a warp per item, all 6
// fields; the items of a level are contiguous.
constexpr int SWEEP_WARPS = 8;

template <typename S, typename GT>
__global__ void __launch_bounds__(SWEEP_WARPS * 32) kin_sweep_kernel(KinSweepParams<S> p)
{
	typedef GT T;
	// per warp: inflow traces [face][field][node] (144), lifted face terms
	// (144), node accumulators (60), right-hand side (60), own f (60), G (100)
	__shared__ __align__(16) T sh[SWEEP_WARPS][144 + 144 + 60 + 60 + 60 + 100];
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	const long long k = (long long)p.item_begin + (long long)blockIdx.x * SWEEP_WARPS + w;
	if (k >= p.item_end)
		return;
	const Tables<T> &tb = tab<T>();
	const int nv = p.nv;
	T *tr = sh[w], *phi = tr + 144, *tacc = phi + 144, *r = tacc + 60, *fs = r + 60, *gs = fs + 60;
	// independent data first, copied asynchronously into shared memory while
	// the trace loads are in flight: own f (60 values) and G (100)
	{
		const S *fe = p.f + k * 60;
		const T *G = reinterpret_cast<const T *>(p.G) + k * 100;
		constexpr int VG = 16 / sizeof(T);
		for (int q = l; q < 100 / VG; q += 32)
			__pipeline_memcpy_async(gs + q * VG, G + q * VG, 16);
		if (sizeof(S) == sizeof(T)) {
			for (int q = l; q < 60 / VG; q += 32)
				__pipeline_memcpy_async(fs + q * VG, reinterpret_cast<const T *>(fe) + q * VG, 16);
		} else {
			for (int q = l; q < 60; q += 32)
				fs[q] = (T)Store<S>::load(fe + q);
		}
		__pipeline_commit();
	}
	const int4 nb4 = p.rnb[k];
	const int4 pm4 = p.rpm[k];
	const int nbk[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
	const int pmk[4] = {pm4.x, pm4.y, pm4.z, pm4.w};
	const T *rs = reinterpret_cast<const T *>(p.rs) + k * 4;
	const int e = p.relem[k];
	const T coef = reinterpret_cast<const T *>(p.coef)[e];
	const int v = p.items[k] % nv;
	// all inflow traces in one round trip: q = (face*6 + field)*6 + node
	for (int q = l; q < 144; q += 32) {
		const int f = q / 36, c = (q % 36) / 6, jj = q % 6;
		const int nbv = f == 0 ? nbk[0] : f == 1 ? nbk[1] : f == 2 ? nbk[2] : nbk[3];
		const int pm = f == 0 ? pmk[0] : f == 1 ? pmk[1] : f == 2 ? pmk[2] : pmk[3];
		T val = T(0);
		if (nbv >= 0) {
			val = (T)Store<S>::load(p.y + (long long)nbv * 60 + c * 10 + ((pm >> (4 * jj)) & 15));
		} else if (nbv != INT_MIN) {
			const double t_half = __dadd_rn(*p.t_dev, __dmul_rn(0.5, p.dt)); // t + dt / 2
			const double *x = p.bxyz + ((long long)(-nbv - 1) * 6 + jj) * 3;
			double xx[3] = {x[0], x[1], x[2]}, we[6], Aw[6];
			exact_w(p.data, xx, t_half, we);
			double n[3] = {p.vi[3 * v], p.vi[3 * v + 1], p.vi[3 * v + 2]};
			maxwell_A<double>(n, we, Aw);
			val = (T)(we[c] / nv + p.feq_c * Aw[c]);
		}
		tr[q] = val;
	}
	__syncwarp();
	// phi[f][c][ii] = s_f (S tr[f][c])_ii on inflow faces
	for (int q = l; q < 144; q += 32) {
		const int f = q / 36, base = q - q % 6, ii = q % 6;
		const int nbv = f == 0 ? nbk[0] : f == 1 ? nbk[1] : f == 2 ? nbk[2] : nbk[3];
		T acc = T(0);
		if (nbv != INT_MIN) {
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				acc += tb.S[ii][jj] * tr[base + jj];
			acc *= rs[f];
		}
		phi[q] = acc;
	}
	__syncwarp();
	// gather the face terms at the element nodes
	for (int q = l; q < 60; q += 32) {
		const int c = q / 10, i = q % 10;
		T acc = T(0);
		for (int a = 0; a < tb.nface_of_node[i]; a++)
			acc += phi[(tb.face_of_node[i][a] * 6 + c) * 6 + tb.pos_of_node[i][a]];
		tacc[q] = acc;
	}
	__pipeline_wait_prior(0);
	__syncwarp();
	for (int q = l; q < 60; q += 32) {
		const int c = q / 10, i = q % 10;
		T acc = T(0);
#pragma unroll
		for (int j = 0; j < 10; j++)
			acc += tb.Minv[i][j] * tacc[c * 10 + j];
		r[q] = fs[q] - coef * acc;
	}
	__syncwarp();
	S *ye = p.y + k * 60;
	for (int q = l; q < 60; q += 32) {
		const int c = q / 10, i = q % 10;
		T acc = T(0);
#pragma unroll
		for (int j = 0; j < 10; j++)
			acc += gs[i * 10 + j] * r[c * 10 + j];
		Store<S>::store(ye + q, acc);
	}
}

template <typename S, typename GT>
int launch_kin_sweep(const KinSweepParams<S> &p, cudaStream_t s)
{
	const long long n = (long long)p.item_end - p.item_begin;
	if (n <= 0)
		return GDN_CUDA_OK;
	kin_sweep_kernel<S, GT><<<(unsigned)((n + SWEEP_WARPS - 1) / SWEEP_WARPS), SWEEP_WARPS * 32, 0, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_sweep<double, double>(const KinSweepParams<double> &, cudaStream_t);
template int launch_kin_sweep<float, float>(const KinSweepParams<float> &, cudaStream_t);

// x = a_y y + a_f f (the Crank-Nicolson transport result), then the
// relaxation of dg_apply_relaxation (dg.c:109-147): w = sum_v x_v,
// f <- omega f_eq(w) + (1 - omega) x.  A thread per (element, node).
template <typename S, typename T, int NV>
__global__ void kin_relax_kernel(KinRelaxParams<S> p)
{
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (t >= p.ne * 10)
		return;
	const long long e = t / 10;
	const int i = (int)(t % 10);
	T x[NV][6], w[6];
	long long base[NV];
#pragma unroll
	for (int c = 0; c < 6; c++)
		w[c] = T(0);
#pragma unroll
	for (int v = 0; v < NV; v++) {
		base[v] = (long long)p.pos[e * NV + v] * 60 + i;
#pragma unroll
		for (int c = 0; c < 6; c++) {
			const long long o = base[v] + c * 10;
			const T xv = (T)p.a_y * (T)Store<S>::load(p.y + o) + (T)p.a_f * (T)Store<S>::load(p.f + o);
			x[v][c] = xv;
			w[c] += xv;
		}
	}
	const T om = (T)p.omega, om1 = T(1) - (T)p.omega, fc = (T)p.feq_c, inv_nv = T(1) / T(NV);
#pragma unroll
	for (int v = 0; v < NV; v++) {
		const T n[3] = {(T)p.vi[3 * v], (T)p.vi[3 * v + 1], (T)p.vi[3 * v + 2]};
		T Aw[6];
		maxwell_A<T>(n, w, Aw);
#pragma unroll
		for (int c = 0; c < 6; c++) {
			const T feq = w[c] * inv_nv + fc * Aw[c];
			Store<S>::store(p.f + base[v] + c * 10, om * feq + om1 * x[v][c]);
		}
	}
}

template <typename S>
int launch_kin_relax(const KinRelaxParams<S> &p, cudaStream_t s)
{
	typedef typename Store<S>::compute T;
	const unsigned nblk = (unsigned)((p.ne * 10 + 255) / 256);
	if (p.nv == 4)
		kin_relax_kernel<S, T, 4><<<nblk, 256, 0, s>>>(p);
	else
		kin_relax_kernel<S, T, 6><<<nblk, 256, 0, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_relax<double>(const KinRelaxParams<double> &, cudaStream_t);
template int launch_kin_relax<float>(const KinRelaxParams<float> &, cudaStream_t);

} // namespace gdn
