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
#include "aux.h"
#include "kernels.h"

namespace gdn {

// own-side v.vn of every element face for every velocity, from the L-side
// normal of each face in the reference's operation order (simulation.c:
// 520-540 + kinetic_num_flux_upwind): the R side gets exactly -s.
template <typename GT>
__global__ void kin_face_s_kernel(const int *__restrict__ face2elem, long long nf, const double *__restrict__ geom,
								  KinModel km, GT *__restrict__ sown, double *__restrict__ sown64)
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
		sown[(eL * km.nv + v) * 4 + fL] = (GT)s;
		sown64[(eL * km.nv + v) * 4 + fL] = s;
		if (eR >= 0) {
			sown[(eR * km.nv + v) * 4 + fR] = (GT)(-s);
			sown64[(eR * km.nv + v) * 4 + fR] = -s;
		}
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

// G = D^-1 per (element, velocity), FP64 Gauss-Jordan with partial pivoting.
template <typename GT>
__global__ void kin_blocks_kernel(const double *__restrict__ geom, const double *__restrict__ sown64, long long ne,
								  KinModel km, double theta_dt, GT *__restrict__ G, GT *__restrict__ coef,
								  int *__restrict__ bad)
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
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++)
			G[u * 100 + i * 10 + j] = (GT)a[i][10 + j];
	if (v == 0)
		coef[e] = (GT)c;
}

template <typename GT>
int launch_kin_setup(const int *face2elem, long long nf, const double *geom, const int *nb, long long ne,
					 const KinModel &km, double theta_dt, GT *sown, double *sown64, unsigned char *mask, GT *G,
					 GT *coef, int *bad, cudaStream_t s)
{
	kin_face_s_kernel<GT><<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(face2elem, nf, geom, km, sown, sown64);
	GDN_CUDA_TRY(cudaGetLastError());
	const long long nu = ne * km.nv;
	kin_mask_kernel<<<(unsigned)((nu + 255) / 256), 256, 0, s>>>(sown64, nb, ne, km.nv, mask);
	GDN_CUDA_TRY(cudaGetLastError());
	kin_blocks_kernel<GT><<<(unsigned)((nu + 127) / 128), 128, 0, s>>>(geom, sown64, ne, km, theta_dt, G, coef,
																	   bad);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_setup<double>(const int *, long long, const double *, const int *, long long,
									  const KinModel &, double, double *, double *, unsigned char *, double *,
									  double *, int *, cudaStream_t);
template int launch_kin_setup<float>(const int *, long long, const double *, const int *, long long,
									 const KinModel &, double, float *, double *, unsigned char *, float *,
									 float *, int *, cudaStream_t);

// One level of the block forward substitution: a warp per (element,
// velocity) item, all 6 fields.
constexpr int SWEEP_WARPS = 8;

template <typename S, typename GT>
__global__ void __launch_bounds__(SWEEP_WARPS * 32) kin_sweep_kernel(KinSweepParams<S> p)
{
	typedef GT T;
	__shared__ T sh[SWEEP_WARPS][3][64];
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	const long long it = (long long)p.item_begin + (long long)blockIdx.x * SWEEP_WARPS + w;
	if (it >= p.item_end)
		return;
	const Tables<T> &tb = tab<T>();
	const int item = p.items[it];
	const int nv = p.nv;
	const long long e = item / nv;
	const int v = item % nv;
	T *tr = sh[w][0], *tacc = sh[w][1], *r = sh[w][2];
	for (int k = l; k < 60; k += 32)
		tacc[k] = T(0);
	__syncwarp();
	const T *sown = reinterpret_cast<const T *>(p.sown) + (e * nv + v) * 4;
	for (int f = 0; f < 4; f++) {
		const T s = sown[f];
		if (!(s < T(0)))
			continue;
		const int nbv = p.nb[e * 4 + f];
		const int pm = p.perm[e * 4 + f];
		for (int k = l; k < 36; k += 32) {
			const int c = k / 6, jj = k % 6;
			T val;
			if (nbv >= 0) {
				const int qn = (pm >> (4 * jj)) & 15;
				val = (T)Store<S>::load(p.y + (((long long)nbv * nv + v) * 6 + c) * 10 + qn);
			} else {
				const double *x = p.bxyz + ((long long)(-nbv - 1) * 6 + jj) * 3;
				double xx[3] = {x[0], x[1], x[2]}, we[6], Aw[6];
				exact_w(p.data, xx, p.t_half, we);
				double n[3] = {p.vi[3 * v], p.vi[3 * v + 1], p.vi[3 * v + 2]};
				maxwell_A<double>(n, we, Aw);
				val = (T)(we[c] / nv + p.feq_c * Aw[c]);
			}
			tr[k] = val;
		}
		__syncwarp();
		for (int k = l; k < 36; k += 32) {
			const int c = k / 6, ii = k % 6;
			T acc = T(0);
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				acc += tb.S[ii][jj] * tr[c * 6 + jj];
			tacc[c * 10 + tb.f2n[f][ii]] += s * acc;
		}
		__syncwarp();
	}
	const T coef = reinterpret_cast<const T *>(p.coef)[e];
	const S *fe = p.f + (e * nv + v) * 60;
	for (int k = l; k < 60; k += 32) {
		const int c = k / 10, i = k % 10;
		T acc = T(0);
#pragma unroll
		for (int j = 0; j < 10; j++)
			acc += tb.Minv[i][j] * tacc[c * 10 + j];
		r[k] = (T)Store<S>::load(fe + k) - coef * acc;
	}
	__syncwarp();
	const T *G = reinterpret_cast<const T *>(p.G) + (e * nv + v) * 100;
	S *ye = p.y + (e * nv + v) * 60;
	for (int k = l; k < 60; k += 32) {
		const int c = k / 10, i = k % 10;
		T acc = T(0);
#pragma unroll
		for (int j = 0; j < 10; j++)
			acc += G[i * 10 + j] * r[c * 10 + j];
		Store<S>::store(ye + k, acc);
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
template <typename S, typename T>
__global__ void kin_relax_kernel(KinRelaxParams<S> p)
{
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (t >= p.ne * 10)
		return;
	const long long e = t / 10;
	const int i = (int)(t % 10);
	const int nv = p.nv;
	T x[NV_MAX][6], w[6];
	for (int c = 0; c < 6; c++)
		w[c] = T(0);
	for (int v = 0; v < nv; v++)
		for (int c = 0; c < 6; c++) {
			const long long o = ((e * nv + v) * 6 + c) * 10 + i;
			const T xv = (T)p.a_y * (T)Store<S>::load(p.y + o) + (T)p.a_f * (T)Store<S>::load(p.f + o);
			x[v][c] = xv;
			w[c] += xv;
		}
	const T om = (T)p.omega, om1 = T(1) - (T)p.omega, fc = (T)p.feq_c, inv_nv = T(1) / T(nv);
	for (int v = 0; v < nv; v++) {
		const T n[3] = {(T)p.vi[3 * v], (T)p.vi[3 * v + 1], (T)p.vi[3 * v + 2]};
		T Aw[6];
		maxwell_A<T>(n, w, Aw);
		for (int c = 0; c < 6; c++) {
			const long long o = ((e * nv + v) * 6 + c) * 10 + i;
			const T feq = w[c] * inv_nv + fc * Aw[c];
			Store<S>::store(p.f + o, om * feq + om1 * x[v][c]);
		}
	}
}

template <typename S>
int launch_kin_relax(const KinRelaxParams<S> &p, cudaStream_t s)
{
	typedef typename Store<S>::compute T;
	kin_relax_kernel<S, T><<<(unsigned)((p.ne * 10 + 255) / 256), 256, 0, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_relax<double>(const KinRelaxParams<double> &, cudaStream_t);
template int launch_kin_relax<float>(const KinRelaxParams<float> &, cudaStream_t);

} // namespace gdn
