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
// it needs in its records (inflow neighbour items, permutations, v . vn,
// theta dt / det).
//
// Mixed precision (GDN_CUDA_FP32_REFINE): FP64 state, FP32 sweeps, FP64
// residual r = f - b - M1 y computed matrix-free from the FP64 geometry, then
// FP32 correction sweeps M1 d = r with zero boundary data, y += d.
#include <climits>
#include <type_traits>

#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
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

__global__ void kin_iota_kernel(int *a, long long n)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u < n)
		a[u] = (int)u;
}

// after the sort: pos = inverse of items, level_off[l] = first item of level l
__global__ void kin_schedule_finish_kernel(const int *__restrict__ items, const int *__restrict__ lev_sorted,
										   long long n, int *__restrict__ pos, int *__restrict__ level_off)
{
	const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (k >= n)
		return;
	pos[items[k]] = (int)k;
	const int l = lev_sorted[k];
	if (k == 0 || lev_sorted[k - 1] != l)
		level_off[l] = (int)k;
	if (k == n - 1)
		level_off[l + 1] = (int)n;
}

static int launch_kin_kahn(const unsigned char *mask, const int *nb, const double *sown64, long long ne, int nv,
						   int *indeg, int *level, int *front0, int *front1, unsigned *ctl, long long spin_limit,
						   cudaStream_t s);

int kin_device_schedule(const unsigned char *mask, const int *nb, const double *sown64, long long ne, int nv,
						int *items, int *pos, std::vector<int> &level_off, long long spin_limit, cudaStream_t s)
{
	const long long nu = ne * nv;
	const unsigned g = (unsigned)((nu + 255) / 256);
	int *level = nullptr, *lev_sorted = nullptr, *iota = nullptr, *indeg = nullptr, *loff = nullptr;
	unsigned *ctl = nullptr;
	void *tmp = nullptr;
	size_t tmp_bytes = 0;
	int rc = GDN_CUDA_OK;
	int maxlev = 0;
	auto cleanup = [&]() {
		cudaFree(level);
		cudaFree(lev_sorted);
		cudaFree(iota);
		cudaFree(indeg);
		cudaFree(ctl);
		cudaFree(loff);
		cudaFree(tmp);
	};
#define GDN_SCHED_TRY(expr)                                                                                           \
	do {                                                                                                           \
		cudaError_t _e = (expr);                                                                                   \
		if (_e != cudaSuccess) {                                                                                   \
			cleanup();                                                                                             \
			return gdn_cuda_fail(_e, #expr, __FILE__, __LINE__);                                                  \
		}                                                                                                          \
	} while (0)
	GDN_SCHED_TRY(cudaMalloc(&level, nu * sizeof(int)));
	GDN_SCHED_TRY(cudaMalloc(&lev_sorted, nu * sizeof(int)));
	GDN_SCHED_TRY(cudaMalloc(&iota, nu * sizeof(int)));
	GDN_SCHED_TRY(cudaMalloc(&indeg, nu * sizeof(int)));
	GDN_SCHED_TRY(cudaMalloc(&ctl, 8 * sizeof(unsigned)));
	GDN_SCHED_TRY(cudaMemsetAsync(ctl, 0, 8 * sizeof(unsigned), s));
	// levels: Kahn's algorithm, the two frontiers in the sort buffers
	{
		const int lrc = launch_kin_kahn(mask, nb, sown64, ne, nv, indeg, level, lev_sorted, iota, ctl, spin_limit, s);
		if (lrc != GDN_CUDA_OK) {
			cleanup();
			return lrc;
		}
		unsigned hctl[8];
		GDN_SCHED_TRY(cudaMemcpyAsync(hctl, ctl, sizeof(hctl), cudaMemcpyDeviceToHost, s));
		GDN_SCHED_TRY(cudaStreamSynchronize(s));
		if (hctl[4]) {
			cleanup();
			return gdn_set_error(GDN_CUDA_ERR_TIMEOUT, "attach: the level schedule's grid barrier timed out");
		}
		if ((long long)hctl[6] != nu) {
			cleanup();
			return gdn_set_error(GDN_CUDA_ERR_CYCLE, "attach: the upwind element graph has a cycle");
		}
	}
	kin_iota_kernel<<<g, 256, 0, s>>>(iota, nu);
	GDN_SCHED_TRY(cudaGetLastError());
	// stable sort of the items by level: within a level the item order is
	// ascending e * nv + v, as the host schedule had it
	int bits = 1;
	{
		int *dmax = reinterpret_cast<int *>(ctl + 7);
		GDN_SCHED_TRY(cub::DeviceReduce::Max(nullptr, tmp_bytes, level, dmax, (int)nu, s));
		GDN_SCHED_TRY(cudaMalloc(&tmp, tmp_bytes));
		GDN_SCHED_TRY(cub::DeviceReduce::Max(tmp, tmp_bytes, level, dmax, (int)nu, s));
		GDN_SCHED_TRY(cudaMemcpyAsync(&maxlev, dmax, sizeof(int), cudaMemcpyDeviceToHost, s));
		GDN_SCHED_TRY(cudaStreamSynchronize(s));
		cudaFree(tmp);
		tmp = nullptr;
		while ((1 << bits) <= maxlev)
			bits++;
	}
	GDN_SCHED_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, level, lev_sorted, iota, items, (int)nu, 0,
												  bits, s));
	GDN_SCHED_TRY(cudaMalloc(&tmp, tmp_bytes));
	GDN_SCHED_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, level, lev_sorted, iota, items, (int)nu, 0, bits,
												  s));
	GDN_SCHED_TRY(cudaMalloc(&loff, (maxlev + 2) * sizeof(int)));
	kin_schedule_finish_kernel<<<g, 256, 0, s>>>(items, lev_sorted, nu, pos, loff);
	GDN_SCHED_TRY(cudaGetLastError());
	level_off.assign(maxlev + 2, 0);
	GDN_SCHED_TRY(cudaMemcpyAsync(level_off.data(), loff, (maxlev + 2) * sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_SCHED_TRY(cudaStreamSynchronize(s));
#undef GDN_SCHED_TRY
	cleanup();
	return rc;
}

// Tables of the block setup, FP64, filled at attach (kin_upload_block_tables):
// MD[d][r][j] = (Minv D_d)[r][j] and MS[f][r][jj] = sum_ii Minv[r][f2n(f, ii)]
// S[ii][jj], so that row r of Minv F is formed from its own row of each.
__constant__ double c_kin_md[3][10][10];
__constant__ double c_kin_ms[4][10][6];

int kin_upload_block_tables(const gdn_cuda_tables *t)
{
	double md[3][10][10], ms[4][10][6];
	for (int d = 0; d < 3; d++)
		for (int r = 0; r < 10; r++)
			for (int j = 0; j < 10; j++) {
				double acc = 0.0;
				for (int k = 0; k < 10; k++)
					acc += t->inv_mass[r][k] * t->internal[k][j][d];
				md[d][r][j] = acc;
			}
	for (int f = 0; f < 4; f++)
		for (int r = 0; r < 10; r++)
			for (int jj = 0; jj < 6; jj++) {
				double acc = 0.0;
				for (int ii = 0; ii < 6; ii++)
					acc += t->inv_mass[r][f2n(f, ii)] * t->face_scal[ii][jj];
				ms[f][r][jj] = acc;
			}
	GDN_CUDA_TRY(cudaMemcpyToSymbol(c_kin_md, md, sizeof(md)));
	GDN_CUDA_TRY(cudaMemcpyToSymbol(c_kin_ms, ms, sizeof(ms)));
	return GDN_CUDA_OK;
}

// G = D^-1 per (element, velocity), FP64 Gauss-Jordan with partial pivoting
// on [D | I], written at the item's sweep position with theta dt / det.
// D = I + c Minv F with F = V + sum_outflow s+ E_f S E_f^T, V_ij = -(v . c_ij),
// row r of Minv F formed directly from the precomputed rows of Minv D_d and
// Minv E_f S.  Ten lanes per item, three items per warp (lanes 30 and 31 idle),
// lane r holding row r of [D | I] in registers (no local memory).
// - Pivot of column k: the largest |a| among the rows not yet used, ties to the
//   smallest position.  A shuffle tree over the item's lanes takes the maximum
//   of |a| as a 64-bit pattern (non-negative doubles order as their bits; +1
//   keeps every candidate above the rows already used); a ballot names the
//   lanes that hold it, and only when two do (anywhere in the warp) a second
//   tree takes the smallest position among them.
// - The normalised pivot row is broadcast through shared memory, and every
//   other row eliminates column k.
// - Rows are not moved: each lane keeps the position its row would have in the
//   row-swapping algorithm, so the pivots are those of the textbook version.
// - Columns left of the pivot are not updated: they no longer feed a pivot or
//   the inverse.
// - The right half is kept in pivot order: slot t holds the column of the row
//   that was the pivot at step t.  Before step k only slots 0..k-1 can differ
//   from the identity (a column of I stays a unit column until its row is a
//   pivot), so step k updates 9 - k left columns and k + 1 slots, and every
//   value equals the one the full [D | I] elimination computes.  The slots go
//   back to their columns when G is written.
constexpr int kBlkThreads = 256;			  // 8 warps, 24 items per CTA
constexpr int kBlkItems = kBlkThreads / 32 * 3;
template <typename GT>
__global__ void __launch_bounds__(kBlkThreads, 4)
	kin_blocks_kernel(const double *__restrict__ geom, const double *__restrict__ sown64,
					  const int *__restrict__ pos, long long ne, KinModel km, double theta,
					  const int *__restrict__ einst, const double *__restrict__ dt_tab, GT *__restrict__ G,
					  GT *__restrict__ rcoef, double4 *__restrict__ ru64, double4 *__restrict__ rs64,
					  int *__restrict__ bad)
{
	__shared__ double sMD[3][10][10], sMS[4][10][6];
	__shared__ __align__(16) double sPiv[kBlkItems][20]; // pivot row of each item
	for (int q = threadIdx.x; q < 300; q += blockDim.x)
		(&sMD[0][0][0])[q] = (&c_kin_md[0][0][0])[q];
	for (int q = threadIdx.x; q < 240; q += blockDim.x)
		(&sMS[0][0][0])[q] = (&c_kin_ms[0][0][0])[q];
	__syncthreads();
	const int lane = threadIdx.x & 31, slot = lane / 10; // slot 3: the two idle lanes
	const bool row = slot < 3;
	const int base = 10 * slot, r = lane - base, seg = row ? 10 : 2;
	const unsigned segmask = row ? 0x3ffu << base : 0xc0000000u;
	const int witem = (threadIdx.x >> 5) * 3 + (row ? slot : 0);
	double *piv = sPiv[witem];
	const long long nu = ne * km.nv;
	const long long u0 = blockIdx.x * (long long)kBlkItems + witem;
	const bool item = row && u0 < nu;
	const long long u = u0 < nu ? u0 : nu - 1; // lanes past the end shadow the last item
	const int rr = row ? r : 0;
	const long long e = u / km.nv;
	const int v = (int)(u % km.nv);
	const double *vv = km.vi + 3 * v;
	double cod[3][3];
#pragma unroll
	for (int a = 0; a < 3; a++)
#pragma unroll
		for (int b = 0; b < 3; b++)
			cod[a][b] = geom[e * 10 + 3 * a + b];
	const double det = geom[e * 10 + 9];
	// u_k = sum_l v_l codtau[l][k]:  v . c_ij = sum_k u_k int d_k phi_i phi_j
	double uk[3];
#pragma unroll
	for (int k = 0; k < 3; k++)
		uk[k] = vv[0] * cod[0][k] + vv[1] * cod[1][k] + vv[2] * cod[2][k];
	double sp[4];
#pragma unroll
	for (int f = 0; f < 4; f++) {
		const double sf = sown64[u * 4 + f];
		sp[f] = sf > 0.0 ? sf : 0.0;
	}
	const double c = theta * dt_tab[einst ? einst[e] : 0] / det;
	const long long kk = pos[u];
	if (item && r == 0) { // the item's records (a singular block fails the attach)
		rcoef[kk] = (GT)c;
		if (ru64) {
			ru64[kk] = make_double4(uk[0], uk[1], uk[2], c);
			rs64[kk] = make_double4(sown64[u * 4], sown64[u * 4 + 1], sown64[u * 4 + 2], sown64[u * 4 + 3]);
		}
	}
	// row rr of [I + c Minv F | I]
	double a[20];
#pragma unroll
	for (int j = 0; j < 10; j++) {
		double acc = -(uk[0] * sMD[0][rr][j] + uk[1] * sMD[1][rr][j] + uk[2] * sMD[2][rr][j]);
#pragma unroll
		for (int f = 0; f < 4; f++)
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				if (f2n(f, jj) == j)
					acc += sp[f] * sMS[f][rr][jj];
		a[j] = (rr == j ? 1.0 : 0.0) + c * acc;
		a[10 + j] = 0.0; // slot j, filled from step j on
	}
	int posn = rr;	// this row's position in the row-swapping algorithm
	unsigned long long col = 0; // 4 bits per step t: the row (= column of I) that was the pivot
	bool singular = false;
#pragma unroll
	for (int k = 0; k < 10; k++) {
		// pivot: the largest |a[k]| among positions >= k, ties to the smallest position
		const bool cand = row && posn >= k;
		const unsigned long long val = cand ? (unsigned long long)__double_as_longlong(fabs(a[k])) + 1ull : 0ull;
		unsigned long long best = val;
#pragma unroll
		for (int off = 1; off < 16; off <<= 1) {
			const int src = r + off < seg ? lane + off : lane;
			const unsigned long long ob = __shfl_sync(0xffffffffu, best, src);
			best = ob > best ? ob : best;
		}
		best = __shfl_sync(0xffffffffu, best, base);
		const unsigned win = __ballot_sync(0xffffffffu, val == best) & segmask;
		int blane = __ffs(win) - 1;
		if (__any_sync(0xffffffffu, row && (win & (win - 1)) != 0)) { // a tie: the smallest position
			int key = val == best ? posn * 32 + lane : 0x7fffffff;
#pragma unroll
			for (int off = 1; off < 16; off <<= 1) {
				const int src = r + off < seg ? lane + off : lane;
				const int ok = __shfl_sync(0xffffffffu, key, src);
				key = ok < key ? ok : key;
			}
			blane = __shfl_sync(0xffffffffu, key, base) & 31;
		}
		const int bpos = __shfl_sync(0xffffffffu, posn, blane);
		col |= (unsigned long long)(blane - base) << (4 * k);
		// the rows at position k and at the pivot's position trade places
		const bool pivot = row && lane == blane;
		if (row && posn == k)
			posn = bpos;
		else if (pivot)
			posn = k;
		if (pivot) {
			if (a[k] == 0.0) {
				singular = true;
			} else {
				const double inv = 1.0 / a[k];
#pragma unroll
				for (int q = k + 1; q < 10; q++) {
					a[q] *= inv;
					piv[q] = a[q];
				}
#pragma unroll
				for (int t = 0; t < k; t++) {
					a[10 + t] *= inv;
					piv[10 + t] = a[10 + t];
				}
				a[10 + k] = inv; // 1 x inv
				piv[10 + k] = inv;
			}
		}
		singular = __shfl_sync(0xffffffffu, (int)singular, blane) != 0 || singular;
		__syncwarp();
		const double m = a[k];
		if (row && lane != blane && m != 0.0) {
#pragma unroll
			for (int q = k + 1; q < 10; q++)
				a[q] -= m * piv[q];
#pragma unroll
			for (int t = 0; t <= k; t++)
				a[10 + t] -= m * piv[10 + t];
		}
		__syncwarp(); // the pivot row is read before the next step overwrites it
	}
	if (!item)
		return;
	if (singular) {
		atomicMax(bad, 1);
		return;
	}
	GT *Gk = G + kk * 100 + posn * 10;
#pragma unroll
	for (int t = 0; t < 10; t++)
		Gk[(col >> (4 * t)) & 15] = (GT)a[10 + t];
}

// per-item records of the sweep
template <typename GT>
__global__ void kin_records_kernel(const int *__restrict__ items, const int *__restrict__ pos,
								   const double *__restrict__ sown64, const int *__restrict__ nb,
								   const int *__restrict__ perm, long long nitems, int nv, int4 *__restrict__ rnb,
								   int4 *__restrict__ rpm, GT *__restrict__ rs)
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
					  const int *perm, long long ne, const KinModel &km, double theta, const int *einst,
					  const double *dt_tab, GT *G, GT *rcoef, int4 *rnb, int4 *rpm, GT *rs, double4 *ru64,
					  double4 *rs64, int *bad, cudaStream_t s)
{
	const long long nu = ne * km.nv;
	kin_blocks_kernel<GT><<<(unsigned)((nu + kBlkItems - 1) / kBlkItems), kBlkThreads, 0, s>>>(
		geom, sown64, pos, ne, km, theta, einst, dt_tab, G, rcoef, ru64, rs64, bad);
	GDN_CUDA_TRY(cudaGetLastError());
	kin_records_kernel<GT><<<(unsigned)((nu + 255) / 256), 256, 0, s>>>(items, pos, sown64, nb, perm, nu, km.nv, rnb,
																		rpm, rs);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_setup<double>(const int *, long long, const double *, const int *, long long,
									  const KinModel &, double *, unsigned char *, cudaStream_t);
template int launch_kin_blocks<double>(const double *, const double *, const int *, const int *, const int *,
									   const int *, long long, const KinModel &, double, const int *, const double *,
									   double *, double *, int4 *, int4 *, double *, double4 *, double4 *, int *,
									   cudaStream_t);
template int launch_kin_blocks<float>(const double *, const double *, const int *, const int *, const int *,
									  const int *, long long, const KinModel &, double, const int *, const double *,
									  float *, float *, int4 *, int4 *, float *, double4 *, double4 *, int *,
									  cudaStream_t);

// f_eq of the analytic data at every boundary face node for every velocity,
// at t + dt/2 (relaxation.c:99, dg_update_boundary with use_feq), formed from
// the device time with the host's rounding.  bt[((bf * nv + v) * 6 + c) * 6 + jj].
__global__ void kin_boundary_trace_kernel(const double *__restrict__ bxyz, long long nbf, Batch b, KinModel km,
										  double *__restrict__ bt)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= nbf * 6)
		return;
	const long long bf = u / 6;
	const int jj = (int)(u % 6);
	const int inst = b.bfinst ? b.bfinst[bf] : 0;
	const double t_half = __dadd_rn(b.t[inst], __dmul_rn(0.5, b.dt[inst]));
	double x[3] = {bxyz[3 * u], bxyz[3 * u + 1], bxyz[3 * u + 2]}, we[6], Aw[6];
	exact_w(b.data[inst], x, t_half, we);
	for (int v = 0; v < km.nv; v++) {
		double n[3] = {km.vi[3 * v], km.vi[3 * v + 1], km.vi[3 * v + 2]};
		maxwell_A<double>(n, we, Aw);
		for (int c = 0; c < 6; c++)
			bt[((bf * km.nv + v) * 6 + c) * 6 + jj] = we[c] / km.nv + km.feq_c * Aw[c];
	}
}

int launch_kin_boundary_trace(const double *bxyz, long long nbf, const Batch &b, int nv, const double *vi,
							  double feq_c, double *bt, cudaStream_t s)
{
	if (nbf <= 0)
		return GDN_CUDA_OK;
	KinModel km;
	km.nv = nv;
	for (int i = 0; i < 3 * NV_MAX; i++)
		km.vi[i] = vi[i];
	km.feq_c = feq_c;
	kin_boundary_trace_kernel<<<(unsigned)((nbf * 6 + 255) / 256), 256, 0, s>>>(bxyz, nbf, b, km, bt);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// 10 consecutive values of one field of one item, converted to T.  The item
// offsets k*60 + c*10 keep float pairs 8-byte, double pairs 16-byte and
// bfloat16 pairs 4-byte aligned.
template <typename S, typename T>
__device__ __forceinline__ void load10(const S *p, T v[10])
{
	if constexpr (std::is_same<S, float>::value) {
		const float2 *q = reinterpret_cast<const float2 *>(p);
#pragma unroll
		for (int i = 0; i < 5; i++) {
			const float2 a = q[i];
			v[2 * i] = (T)a.x;
			v[2 * i + 1] = (T)a.y;
		}
	} else if constexpr (std::is_same<S, double>::value) {
		const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
		for (int i = 0; i < 5; i++) {
			const double2 a = q[i];
			v[2 * i] = (T)a.x;
			v[2 * i + 1] = (T)a.y;
		}
	} else {
		const __nv_bfloat162 *q = reinterpret_cast<const __nv_bfloat162 *>(p);
#pragma unroll
		for (int i = 0; i < 5; i++) {
			const float2 a = __bfloat1622float2(q[i]);
			v[2 * i] = (T)a.x;
			v[2 * i + 1] = (T)a.y;
		}
	}
}

template <typename S, typename T>
__device__ __forceinline__ void store10(S *p, const T v[10])
{
	if constexpr (std::is_same<S, float>::value) {
		float2 *q = reinterpret_cast<float2 *>(p);
#pragma unroll
		for (int i = 0; i < 5; i++)
			q[i] = make_float2((float)v[2 * i], (float)v[2 * i + 1]);
	} else if constexpr (std::is_same<S, double>::value) {
		double2 *q = reinterpret_cast<double2 *>(p);
#pragma unroll
		for (int i = 0; i < 5; i++)
			q[i] = make_double2((double)v[2 * i], (double)v[2 * i + 1]);
	} else {
		__nv_bfloat162 *q = reinterpret_cast<__nv_bfloat162 *>(p);
#pragma unroll
		for (int i = 0; i < 5; i++)
			q[i] = __floats2bfloat162_rn((float)v[2 * i], (float)v[2 * i + 1]);
	}
}

// One level of the block forward substitution.  A CTA takes 32 consecutive
// items of the level with 6 warps: lane = item, warp = field, so the tables
// are warp-uniform (constant-bank operands) and every thread owns one field
// of one item end to end:
//   traces of the inflow faces (24 independent loads, one round trip),
//   t = sum_inflow s E_f S tr_f,  r = f - coef Minv t,  y = G r.
// G of the 32 items is staged by cp.async into shared memory while the
// traces are in flight; its per-item stride (100 floats / 102 doubles) keeps
// the 16-byte row reads conflict-free.  Levels are launched with programmatic
// stream serialization: level l + 1 stages G, records and f while level l
// runs, and waits (griddepcontrol.wait) only before its trace loads.
constexpr int kSwItems = 32;
constexpr int kSwThreads = 6 * 32;

template <typename T>
struct SweepG {
	static constexpr int stride = sizeof(T) == 4 ? 100 : 102;
	typedef typename std::conditional<sizeof(T) == 4, float4, double2>::type vec;
	static constexpr int per_vec = 16 / sizeof(T);
};

// A chunk: up to 32 items of one level, [k0, min(k0 + 32, item_end)), or with
// `list` the items list[k0 .. item_end).  Lane = item, warp = field c.  It is
// processed in three pieces:
//   chunk_stage_G  G of the chunk's items into shared memory (cp.async, one
//                  commit group);
//   chunk_load     the thread's records, right-hand side and FP64
//                  accumulator into registers (data no sweep step writes);
//   chunk_solve    traces of the upwind neighbours, t = sum_inflow s E S tr,
//                  r = f - coef Minv t, then (after its G group has landed and
//                  a barrier) y = G r and the stores, and a closing barrier.
// Between chunk_load and chunk_solve the caller waits for the upwind items the
// chunk depends on.  L2 = true reads the traces through L2 only (L1 is not
// coherent with other SMs' writes made during the same launch); FENCE = true
// orders every thread's y stores device-wide before the closing barrier;
// WAITG = cp.async groups committed after this chunk's G (0 or 1).
template <typename T, int ACC>
struct ChunkIn {
	long long k;
	int nloc;
	bool act;
	int nbk[4], pmk[4];
	T fv[10];
	double ya[ACC == 2 ? 10 : 1];
	T coef;
	T s[4];
	int v;
};

__device__ __forceinline__ int chunk_nloc(long long k0, long long item_end)
{
	const long long rem = item_end - k0;
	return rem < kSwItems ? (int)rem : kSwItems;
}

template <typename T>
__device__ __forceinline__ void chunk_stage_G(const KinSweepParams &p, long long k0, int nloc, const int *list, T *gsh)
{
	typedef SweepG<T> SG;
	constexpr int VPC = SG::per_vec, CH = 100 / VPC;
	const T *G = reinterpret_cast<const T *>(p.G);
	for (int q = threadIdx.x; q < nloc * CH; q += kSwThreads) {
		const int it = q / CH, ch = q - it * CH;
		const long long kit = list ? (long long)list[k0 + it] : k0 + it;
		__pipeline_memcpy_async(gsh + it * SG::stride + ch * VPC, G + kit * 100 + ch * VPC, 16);
	}
	__pipeline_commit();
}

template <typename F, typename T, int ACC, bool BD>
__device__ __forceinline__ void chunk_load(const KinSweepParams &p, long long k0, long long item_end, const int *list,
										   ChunkIn<T, ACC> &in)
{
	const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
	in.nloc = chunk_nloc(k0, item_end);
	in.act = lane < in.nloc;
	const long long k = list ? (long long)list[k0 + (in.act ? lane : 0)] : k0 + (in.act ? lane : 0);
	in.k = k;
	const int4 nb4 = p.rnb[k];
	const int4 pm4 = p.rpm[k];
	in.nbk[0] = nb4.x, in.nbk[1] = nb4.y, in.nbk[2] = nb4.z, in.nbk[3] = nb4.w;
	in.pmk[0] = pm4.x, in.pmk[1] = pm4.y, in.pmk[2] = pm4.z, in.pmk[3] = pm4.w;
	load10<F, T>(reinterpret_cast<const F *>(p.f) + k * 60 + c * 10, in.fv);
	if (ACC == 2)
		load10<double, double>(p.yacc + k * 60 + c * 10, in.ya);
	in.coef = reinterpret_cast<const T *>(p.rcoef)[k];
	const T *rs = reinterpret_cast<const T *>(p.rs) + k * 4;
#pragma unroll
	for (int f = 0; f < 4; f++)
		in.s[f] = rs[f];
	in.v = BD ? p.items[k] % p.nv : 0;
}

template <typename F, typename Y, typename T, int ACC, bool BD, bool SPARSE, bool L2, bool FENCE, int WAITG>
__device__ __forceinline__ void chunk_solve(const KinSweepParams &p, const ChunkIn<T, ACC> &in, T *gsh)
{
	typedef SweepG<T> SG;
	const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
	const Tables<T> &tb = tab<T>();
	const long long k = in.k;
	T r[10];
	{
		T tr[4][6];
#pragma unroll
		for (int f = 0; f < 4; f++) {
			const int nbv = in.nbk[f];
			if (nbv >= 0) {
				const Y *yn = reinterpret_cast<const Y *>(p.y) + (long long)nbv * 60 + c * 10;
#pragma unroll
				for (int jj = 0; jj < 6; jj++) {
					const Y *q = yn + ((in.pmk[f] >> (4 * jj)) & 15);
					tr[f][jj] = (T)(L2 ? Store<Y>::load_l2(q) : Store<Y>::load(q));
				}
			} else if (BD && nbv != INT_MIN) {
				const double *b = p.bt + (((long long)(-nbv - 1) * p.nv + in.v) * 6 + c) * 6;
#pragma unroll
				for (int jj = 0; jj < 6; jj++)
					tr[f][jj] = (T)b[jj];
			} else {
#pragma unroll
				for (int jj = 0; jj < 6; jj++)
					tr[f][jj] = T(0);
			}
		}
		// t_i = sum over the faces through node i of s_f (S tr_f)_ii
		T t[10];
#pragma unroll
		for (int i = 0; i < 10; i++)
			t[i] = T(0);
#pragma unroll
		for (int f = 0; f < 4; f++) {
#pragma unroll
			for (int ii = 0; ii < 6; ii++) {
				T acc = T(0);
#pragma unroll
				for (int jj = 0; jj < 6; jj++)
					if (!SPARSE || (smask(ii) >> jj & 1))
						acc += tb.S[ii][jj] * tr[f][jj];
				t[f2n(f, ii)] += acc * in.s[f];
			}
		}
#pragma unroll
		for (int i = 0; i < 10; i++) {
			T acc = T(0);
#pragma unroll
			for (int j = 0; j < 10; j++)
				acc += tb.Minv[i][j] * t[j];
			r[i] = in.fv[i] - in.coef * acc;
		}
	}
	__pipeline_wait_prior(WAITG);
	__syncthreads();
	if (in.act) {
		T y[10];
#pragma unroll
		for (int i = 0; i < 10; i++)
			y[i] = T(0);
		const typename SG::vec *g = reinterpret_cast<const typename SG::vec *>(gsh + lane * SG::stride);
#pragma unroll
		for (int q = 0; q < 100 / SG::per_vec; q++) {
			const typename SG::vec gv = g[q];
			const T *ge = reinterpret_cast<const T *>(&gv);
#pragma unroll
			for (int u = 0; u < SG::per_vec; u++) {
				const int idx = q * SG::per_vec + u;
				y[idx / 10] += ge[u] * r[idx % 10];
			}
		}
		store10<Y, T>(reinterpret_cast<Y *>(p.y) + k * 60 + c * 10, y);
		if (ACC == 1) {
			store10<double, T>(p.yacc + k * 60 + c * 10, y);
		} else if (ACC == 2) {
			double ya[10];
#pragma unroll
			for (int i = 0; i < 10; i++)
				ya[i] = in.ya[i] + (double)y[i];
			store10<double, double>(p.yacc + k * 60 + c * 10, ya);
		}
	}
	if (FENCE)
		__threadfence();
	// gsh is reused by the CTA's next chunk
	__syncthreads();
}

// One chunk, start to end.  `wait` is called by every thread between the
// loads and the solve, with its item's inflow records nbk[4] (item index >= 0
// for an upwind neighbour), its permutation records pmk[4] and whether the
// thread holds an item.
template <typename F, typename Y, typename T, int ACC, bool BD, bool SPARSE, bool L2, bool FENCE, typename Wait>
__device__ __forceinline__ void sweep_chunk(const KinSweepParams &p, long long k0, long long item_end, T *gsh,
											Wait wait, const int *list = nullptr)
{
	chunk_stage_G<T>(p, k0, chunk_nloc(k0, item_end), list, gsh);
	ChunkIn<T, ACC> in;
	chunk_load<F, T, ACC, BD>(p, k0, item_end, list, in);
	wait(in.nbk, in.pmk, in.act);
	chunk_solve<F, Y, T, ACC, BD, SPARSE, L2, FENCE, 0>(p, in, gsh);
}

template <typename F, typename Y, typename T, int ACC, bool BD, bool SPARSE>
__global__ void __launch_bounds__(kSwThreads) kin_sweep_kernel(KinSweepParams p)
{
	__shared__ __align__(16) T gsh[kSwItems * SweepG<T>::stride];
	// Programmatic dependent launch: the next level's CTAs may start now and
	// run their prologue (everything before griddepcontrol.wait reads only
	// data that no sweep level writes).
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
	const long long k0 = (long long)p.item_begin + (long long)blockIdx.x * kSwItems;
	// the upwind items of earlier levels are complete once the previous
	// level's grid is
	sweep_chunk<F, Y, T, ACC, BD, SPARSE, false, false>(
		p, k0, p.item_end, gsh, [](const int *, const int *, bool) { asm volatile("griddepcontrol.wait;" ::: "memory"); });
}

// Grid-wide barrier of a cooperative launch (all CTAs co-resident).  *count
// only grows during the launch (it is cleared before the launch): barrier j
// is passed once it reaches (j + 1) x gridDim.x arrivals.  Arrivals are
// release-ordered, polls acquire-ordered.  The wait is bounded: after
// spin_limit polls the CTA sets *err and leaves, and so does every other CTA
// once it sees *err, so a lost CTA ends the launch instead of hanging it.
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned target, int *err, long long spin_limit)
{
	__shared__ int s_ok;
	__syncthreads();
	if (threadIdx.x == 0) {
		volatile int *verr = err;
		int ok = 1;
		asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
		long long it = 0;
		for (;;) {
			unsigned v;
			asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
			if (v >= target)
				break;
			if (*verr || ++it > spin_limit) {
				atomicExch(err, 1);
				ok = 0;
				break;
			}
			__nanosleep(16);
		}
		s_ok = ok && !*verr;
	}
	__syncthreads();
	return s_ok != 0;
}

// Level schedule by Kahn's algorithm, one level per grid barrier, in one
// cooperative launch.  indeg[u] = the upwind dependencies of item u not yet
// placed; the items of level l are listed in one frontier, and placing one
// releases its downwind items (across the faces it flows out of: s > 0 there,
// s < 0 on the other side, so each dependency edge is counted once on each
// end).  An item whose last dependency is placed at level l enters level
// l + 1, so level(u) = the longest upwind chain ending at u.  ctl: [0] barrier
// arrivals, [1..3] frontier sizes of levels l mod 3, [4] error, [5] levels,
// [6] items placed (fewer than all: a cycle).
constexpr int kKahnThreads = 512; // one CTA per SM: the barrier's arrivals, not the work, set a level's time
__global__ void __launch_bounds__(kKahnThreads)
	kin_kahn_kernel(const unsigned char *__restrict__ mask, const int *__restrict__ nb,
					const double *__restrict__ sown64, long long ne, int nv, int *__restrict__ indeg,
					int *__restrict__ level, int *front0, int *front1, unsigned *ctl, long long spin_limit)
{
	const long long nu = ne * nv;
	const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	const long long nthreads = (long long)gridDim.x * blockDim.x;
	const int lane = threadIdx.x & 31;
	const unsigned lt = (1u << lane) - 1u;
	unsigned *bar = ctl, *cnt = ctl + 1;
	int *err = reinterpret_cast<int *>(ctl + 4);
	// level 0: the items without upwind dependencies (warp-aggregated appends)
	for (long long b = tid - lane; b < nu; b += nthreads) {
		const long long u = b + lane;
		int d = 0;
		if (u < nu) {
			d = __popc(mask[u]);
			indeg[u] = d;
		}
		const bool push = u < nu && d == 0;
		const unsigned bal = __ballot_sync(0xffffffffu, push);
		unsigned base = 0;
		if (lane == 0 && bal)
			base = atomicAdd(cnt, __popc(bal));
		base = __shfl_sync(0xffffffffu, base, 0);
		if (push) {
			front0[base + __popc(bal & lt)] = (int)u;
			level[u] = 0;
		}
	}
	if (!grid_barrier(bar, gridDim.x, err, spin_limit))
		return;
	int *cur = front0, *nxt = front1;
	long long placed = 0;
	int l = 0;
	for (;; l++) {
		const unsigned n = *(volatile unsigned *)(cnt + l % 3);
		if (n == 0)
			break;
		placed += n;
		if (tid == 0)
			cnt[(l + 2) % 3] = 0; // level l - 1's size: read by every CTA before the last barrier
		for (long long b = tid - lane; b < n; b += nthreads) {
			const long long i = b + lane;
			const long long u = i < n ? cur[i] : 0;
			const long long e = u / nv;
			const int v = (int)(u % nv);
#pragma unroll
			for (int f = 0; f < 4; f++) {
				bool push = false;
				int w = 0;
				if (i < n) {
					const int we = nb[e * 4 + f];
					if (we >= 0 && sown64[u * 4 + f] > 0.0) {
						w = (int)((long long)we * nv + v);
						push = atomicSub(indeg + w, 1) == 1;
					}
				}
				const unsigned bal = __ballot_sync(0xffffffffu, push);
				unsigned base = 0;
				if (lane == 0 && bal)
					base = atomicAdd(cnt + (l + 1) % 3, __popc(bal));
				base = __shfl_sync(0xffffffffu, base, 0);
				if (push) {
					nxt[base + __popc(bal & lt)] = w;
					level[w] = l + 1;
				}
			}
		}
		if (!grid_barrier(bar, (unsigned)(l + 2) * gridDim.x, err, spin_limit))
			return;
		int *t = cur;
		cur = nxt;
		nxt = t;
	}
	if (tid == 0) {
		ctl[5] = (unsigned)l;
		ctl[6] = (unsigned)placed;
	}
}

// cooperative launch of kin_kahn_kernel with every CTA resident
static int launch_kin_kahn(const unsigned char *mask, const int *nb, const double *sown64, long long ne, int nv,
						   int *indeg, int *level, int *front0, int *front1, unsigned *ctl, long long spin_limit,
						   cudaStream_t s)
{
	int dev = 0, nsm = 0, per = 0;
	GDN_CUDA_TRY(cudaGetDevice(&dev));
	GDN_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
	GDN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kin_kahn_kernel, kKahnThreads, 0));
	if (per < 1)
		return gdn_set_error(GDN_CUDA_ERR_CUDA, "attach: the level schedule kernel cannot be resident");
	const long long nu = ne * nv;
	long long grid = nsm;
	const long long need = (nu + kKahnThreads - 1) / kKahnThreads;
	if (grid > need)
		grid = need;
	if (grid < 1)
		grid = 1;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)grid);
	cfg.blockDim = dim3(kKahnThreads);
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	GDN_CUDA_TRY(cudaLaunchKernelEx(&cfg, kin_kahn_kernel, mask, nb, sown64, ne, nv, indeg, level, front0, front1,
									ctl, spin_limit));
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// All levels of one transport solve in one cooperative launch: the CTAs walk
// the levels in order, 32 items per chunk, with a grid barrier between levels.
// A CTA stages its first chunk of level l (G, records, right-hand side) before
// it waits at the barrier that ends level l - 1.
template <typename F, typename Y, typename T, int ACC, bool BD, bool SPARSE>
__global__ void __launch_bounds__(kSwThreads) kin_levels_kernel(KinSweepParams p, const int *__restrict__ level_off,
																	int nlevels, unsigned *bar, int *err,
																	long long spin_limit)
{
	__shared__ __align__(16) T gsh[kSwItems * SweepG<T>::stride];
	for (int l = 0; l < nlevels; l++) {
		const long long b = level_off[l], e = level_off[l + 1];
		const long long nch = (e - b + kSwItems - 1) / kSwItems;
		bool pending = l > 0; // the barrier ending level l - 1 is still to pass
		bool ok = true;
		const unsigned target = (unsigned)l * gridDim.x;
		for (long long ch = blockIdx.x; ch < nch; ch += gridDim.x) {
			sweep_chunk<F, Y, T, ACC, BD, SPARSE, true, false>(p, b + ch * kSwItems, e, gsh, [&](const int *, const int *, bool) {
				if (pending) {
					ok = grid_barrier(bar, target, err, spin_limit);
					pending = false;
				}
			});
			if (!ok)
				return;
		}
		if (pending && !grid_barrier(bar, target, err, spin_limit))
			return;
	}
}

// Bounded wait for the readiness flags of an item's upwind neighbours
// (need[f]): the flags are polled together with relaxed loads, and once all
// are set one acquire fence orders the caller's later loads after the
// producers' releases (the acquire pattern).  false when *err is set by
// another CTA, or after spin_limit further polls (then *err is set here), so
// a lost producer ends the launch instead of hanging it.  Only warp 0 of a CTA
// waits; acquire loads one flag after another cost up to three L2 round trips
// when the flags are already set.
__device__ __forceinline__ bool wait_ready_all(const int *ready, const int nbk[4], const bool need[4], int *err,
											   long long spin_limit)
{
	bool ok[4];
#pragma unroll
	for (int f = 0; f < 4; f++)
		ok[f] = !need[f];
	const volatile int *verr = err;
	for (long long it = 0;; it++) {
		int v[4];
#pragma unroll
		for (int f = 0; f < 4; f++) {
			v[f] = 1;
			if (!ok[f])
				asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v[f]) : "l"(ready + nbk[f]) : "memory");
		}
		bool all = true;
#pragma unroll
		for (int f = 0; f < 4; f++) {
			ok[f] = ok[f] || v[f] != 0;
			all = all && ok[f];
		}
		if (all)
			break;
		if (*verr)
			return false;
		if (it >= spin_limit) {
			atomicExch(err, 1);
			return false;
		}
		if (it >= 32)
			__nanosleep(32);
	}
	asm volatile("fence.acq_rel.gpu;" ::: "memory");
	return true;
}

// The whole transport solve in one launch, driven by per-item readiness flags
// instead of a barrier per level.  chunks[] lists the solve's 32-item chunks
// in sweep order, never straddling a level, so every upwind item of a chunk
// lies in an earlier chunk.  Each CTA takes the next chunk from an atomic
// counter, stages it, waits (acquire, warp 0 only: a barrier then orders
// the other warps' loads) for the flags of its own items' upwind neighbours,
// solves, and publishes its items' flags (release).  A
// chunk waits only on chunks taken earlier by CTAs already running, so the
// solve progresses with any number of resident CTAs; the critical path is the
// longest upwind chain, not the level count times a launch.  A CTA takes its
// next ticket while it works on the current chunk (the smallest unfinished
// chunk is still always being worked on).  Publication follows the barrier +
// one release store pattern: the chunk's closing barrier orders every warp's
// y stores before the release stores of the flags.  ready[] (one int per item)
// and *queue are zero at launch.
template <typename F, typename Y, typename T, int ACC, bool BD, bool SPARSE>
__global__ void __launch_bounds__(kSwThreads)
	kin_flags_kernel(KinSweepParams p, const int2 *__restrict__ chunks, int nchunks, unsigned *queue, int *ready,
					 int *err, long long spin_limit)
{
	__shared__ __align__(16) T gsh[kSwItems * SweepG<T>::stride];
	__shared__ int s_chunk, s_fail;
	int next = 0; // thread 0: the ticket taken ahead
	if (threadIdx.x == 0)
		next = (int)atomicAdd(queue, 1u);
	for (;;) {
		__syncthreads(); // the previous chunk's s_chunk / s_fail have been read
		if (threadIdx.x == 0) {
			s_chunk = next;
			s_fail = 0;
		}
		__syncthreads();
		const int c = s_chunk;
		if (c >= nchunks)
			return;
		if (threadIdx.x == 0)
			next = (int)atomicAdd(queue, 1u);
		const int2 ck = chunks[c];
		sweep_chunk<F, Y, T, ACC, BD, SPARSE, true, false>(
			p, ck.x, ck.y, gsh, [&](const int *nbk, const int *, bool act) {
				// warp 0 waits for the chunk; the barrier orders the other
				// warps' trace loads after its acquires
				if (threadIdx.x < 32 && act) {
					bool need[4];
#pragma unroll
					for (int f = 0; f < 4; f++)
						need[f] = nbk[f] >= 0;
					if (!wait_ready_all(ready, nbk, need, err, spin_limit))
						s_fail = 1;
				}
				__syncthreads();
			});
		// sweep_chunk ended with a barrier after every thread's y stores
		if (s_fail)
			return; // *err is set; the state of this solve is invalid
		if (threadIdx.x < ck.y - ck.x)
			asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(ready + ck.x + threadIdx.x), "r"(1)
						 : "memory");
	}
}

// The whole transport solve in one cooperative launch, each CTA sweeping one
// spatial part of the mesh.  Elements are split into compact parts (equal
// ranges along a Morton curve of their centroids; all velocities of an element
// in one part), and part b's items are listed in sweep order in plist[], cut
// into chunks (pchunks[c] = first list position, count) that never straddle a
// level.  CTA b walks its chunks in order, so an upwind item in its own part
// was solved by an earlier chunk of the same CTA (the chunk's closing barrier
// orders it); only an upwind item of another part, marked by bit 28 of the
// face's permutation record, is waited for through its readiness flag
// (acquire), and every chunk publishes its items' flags (release).  All CTAs
// are co-resident (cooperative launch), and the unfinished item of lowest
// level always belongs to a chunk whose part is working on it, so the solve
// progresses; the waits are bounded as in the flag-driven sweep.  Inside a
// part a dependent step costs one chunk (a barrier, traces through L2, the
// block solve) instead of one launch per level.
constexpr int kPartExternal = 1 << 28;
template <typename F, typename Y, typename T, int ACC, bool BD, bool SPARSE>
__global__ void __launch_bounds__(kSwThreads)
	kin_parts_kernel(KinSweepParams p, const int *__restrict__ plist, const int2 *__restrict__ pchunks,
					 const int *__restrict__ part_chunk_off, int *ready, int *err, long long spin_limit)
{
	__shared__ __align__(16) T gsh[kSwItems * SweepG<T>::stride];
	__shared__ int s_fail;
	if (threadIdx.x == 0)
		s_fail = 0;
	__syncthreads();
	const int c_end = part_chunk_off[blockIdx.x + 1];
	for (int c = part_chunk_off[blockIdx.x]; c < c_end; c++) {
		const int2 ck = pchunks[c];
		sweep_chunk<F, Y, T, ACC, BD, SPARSE, true, false>(
			p, ck.x, ck.x + ck.y, gsh,
			[&](const int *nbk, const int *pmk, bool act) {
				if (threadIdx.x < 32 && act) {
					bool need[4];
#pragma unroll
					for (int f = 0; f < 4; f++)
						need[f] = nbk[f] >= 0 && (pmk[f] & kPartExternal);
					if (!wait_ready_all(ready, nbk, need, err, spin_limit))
						s_fail = 1;
				}
				__syncthreads();
			},
			plist);
		// sweep_chunk ended with a barrier after every thread's y stores
		if (s_fail)
			return; // *err is set; the state of this solve is invalid
		if (threadIdx.x < ck.y)
			asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(ready + plist[ck.x + threadIdx.x]), "r"(1)
						 : "memory");
	}
}

// Morton code (10 bits per axis) of each element's vertex centroid in the box
// [lo, lo + 1 / inv_ext)
__device__ __forceinline__ unsigned spread10(unsigned x)
{
	x &= 1023u;
	x = (x | (x << 16)) & 0x030000FFu;
	x = (x | (x << 8)) & 0x0300F00Fu;
	x = (x | (x << 4)) & 0x030C30C3u;
	x = (x | (x << 2)) & 0x09249249u;
	return x;
}
__global__ void kin_morton_kernel(const int *__restrict__ e2q, const double *__restrict__ node, long long ne,
								  double3 lo, double3 inv_ext, unsigned *__restrict__ code, int *__restrict__ elem)
{
	const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (e >= ne)
		return;
	double c[3] = {0.0, 0.0, 0.0};
	for (int i = 0; i < 4; i++)
		for (int a = 0; a < 3; a++)
			c[a] += 0.25 * node[3LL * e2q[10 * e + i] + a];
	const double l[3] = {lo.x, lo.y, lo.z}, s[3] = {inv_ext.x, inv_ext.y, inv_ext.z};
	unsigned q[3];
	for (int a = 0; a < 3; a++) {
		const double t = (c[a] - l[a]) * s[a] * 1024.0;
		q[a] = t <= 0.0 ? 0u : (t >= 1023.0 ? 1023u : (unsigned)t);
	}
	code[e] = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
	elem[e] = (int)e;
}
// part of each element from its rank along the curve; part of each item
__global__ void kin_part_of_elem_kernel(const int *__restrict__ elem_sorted, long long ne, int nparts,
										int *__restrict__ part_of_elem)
{
	const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (r < ne)
		part_of_elem[elem_sorted[r]] = (int)(r * nparts / ne);
}
__global__ void kin_part_of_item_kernel(const int *__restrict__ items, const int *__restrict__ part_of_elem,
										long long nitems, int nv, int *__restrict__ part_key, int *__restrict__ iota)
{
	const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (k >= nitems)
		return;
	part_key[k] = part_of_elem[items[k] / nv];
	iota[k] = (int)k;
}
// bit 28 of rpm[k].f: the upwind item across face f belongs to another part
__global__ void kin_mark_external_kernel(const int4 *__restrict__ rnb, const int *__restrict__ part_of_item,
										 long long nitems, int4 *__restrict__ rpm)
{
	const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (k >= nitems)
		return;
	const int4 nb = rnb[k];
	int4 pm = rpm[k];
	const int me = part_of_item[k];
	const int n[4] = {nb.x, nb.y, nb.z, nb.w};
	int m[4] = {pm.x & ~kPartExternal, pm.y & ~kPartExternal, pm.z & ~kPartExternal, pm.w & ~kPartExternal};
	for (int f = 0; f < 4; f++)
		if (n[f] >= 0 && part_of_item[n[f]] != me)
			m[f] |= kPartExternal;
	rpm[k] = make_int4(m[0], m[1], m[2], m[3]);
}

// Spatial parts of the item list (kin_parts_kernel): nparts compact element
// parts; on return plist (device, [nitems]: items of part 0 in sweep order,
// then part 1, ...), pkey_host (host, [nitems]: the part of plist[i]) and the
// external-dependency bits of rpm are set.
int kin_build_parts(const int *e2q, const double *node, long long ne, const double lo[3], const double hi[3],
					const int *items, long long nitems, int nv, int nparts, const int4 *rnb, int4 *rpm, int *plist,
					std::vector<int> &plist_host, std::vector<int> &pkey_host, cudaStream_t s)
{
	unsigned *code = nullptr, *code_s = nullptr;
	int *elem = nullptr, *elem_s = nullptr, *pe = nullptr, *pkey = nullptr, *pkey_s = nullptr, *iota = nullptr;
	void *tmp = nullptr;
	size_t tb = 0, tb2 = 0;
	auto cleanup = [&]() {
		cudaFree(code);
		cudaFree(code_s);
		cudaFree(elem);
		cudaFree(elem_s);
		cudaFree(pe);
		cudaFree(pkey);
		cudaFree(pkey_s);
		cudaFree(iota);
		cudaFree(tmp);
	};
#define GDN_PARTS_TRY(expr)                                                                                           \
	do {                                                                                                           \
		cudaError_t _e = (expr);                                                                                   \
		if (_e != cudaSuccess) {                                                                                   \
			cleanup();                                                                                             \
			return gdn_cuda_fail(_e, #expr, __FILE__, __LINE__);                                                  \
		}                                                                                                          \
	} while (0)
	GDN_PARTS_TRY(cudaMalloc(&code, ne * sizeof(unsigned)));
	GDN_PARTS_TRY(cudaMalloc(&code_s, ne * sizeof(unsigned)));
	GDN_PARTS_TRY(cudaMalloc(&elem, ne * sizeof(int)));
	GDN_PARTS_TRY(cudaMalloc(&elem_s, ne * sizeof(int)));
	GDN_PARTS_TRY(cudaMalloc(&pe, ne * sizeof(int)));
	GDN_PARTS_TRY(cudaMalloc(&pkey, nitems * sizeof(int)));
	GDN_PARTS_TRY(cudaMalloc(&pkey_s, nitems * sizeof(int)));
	GDN_PARTS_TRY(cudaMalloc(&iota, nitems * sizeof(int)));
	double3 l = make_double3(lo[0], lo[1], lo[2]), ie;
	ie.x = 1.0 / (hi[0] - lo[0] > 0.0 ? hi[0] - lo[0] : 1.0);
	ie.y = 1.0 / (hi[1] - lo[1] > 0.0 ? hi[1] - lo[1] : 1.0);
	ie.z = 1.0 / (hi[2] - lo[2] > 0.0 ? hi[2] - lo[2] : 1.0);
	const unsigned ge = (unsigned)((ne + 255) / 256), gi = (unsigned)((nitems + 255) / 256);
	kin_morton_kernel<<<ge, 256, 0, s>>>(e2q, node, ne, l, ie, code, elem);
	GDN_PARTS_TRY(cudaGetLastError());
	GDN_PARTS_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, code, code_s, elem, elem_s, (int)ne, 0, 30, s));
	GDN_PARTS_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb2, pkey, pkey_s, iota, plist, (int)nitems, 0, 31, s));
	GDN_PARTS_TRY(cudaMalloc(&tmp, tb > tb2 ? tb : tb2));
	tb = tb > tb2 ? tb : tb2;
	GDN_PARTS_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, code, code_s, elem, elem_s, (int)ne, 0, 30, s));
	kin_part_of_elem_kernel<<<ge, 256, 0, s>>>(elem_s, ne, nparts, pe);
	GDN_PARTS_TRY(cudaGetLastError());
	kin_part_of_item_kernel<<<gi, 256, 0, s>>>(items, pe, nitems, nv, pkey, iota);
	GDN_PARTS_TRY(cudaGetLastError());
	kin_mark_external_kernel<<<gi, 256, 0, s>>>(rnb, pkey, nitems, rpm);
	GDN_PARTS_TRY(cudaGetLastError());
	int bits = 1;
	while ((1 << bits) <= nparts)
		bits++;
	// stable: within a part the items keep their sweep order
	GDN_PARTS_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, pkey, pkey_s, iota, plist, (int)nitems, 0, bits, s));
	plist_host.resize(nitems);
	pkey_host.resize(nitems);
	GDN_PARTS_TRY(cudaMemcpyAsync(plist_host.data(), plist, nitems * sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_PARTS_TRY(cudaMemcpyAsync(pkey_host.data(), pkey_s, nitems * sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_PARTS_TRY(cudaStreamSynchronize(s));
#undef GDN_PARTS_TRY
	cleanup();
	return GDN_CUDA_OK;
}

template <typename F, typename Y, typename T>
int launch_kin_parts(const KinSweepParams &p, const int *plist, const int2 *pchunks, const int *part_chunk_off,
					 int nparts, int *ready, long long nitems, int *err, long long spin, int acc, int bdata,
					 int sparse, cudaStream_t s)
{
	if (nparts <= 0)
		return GDN_CUDA_OK;
	GDN_CUDA_TRY(cudaMemsetAsync(ready, 0, (size_t)nitems * sizeof(int), s));
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)nparts);
	cfg.blockDim = dim3(kSwThreads);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
#define GDN_PARTS(A, B, SP)                                                                                           \
	GDN_CUDA_TRY(cudaLaunchKernelEx(&cfg, kin_parts_kernel<F, Y, T, A, B, SP>, p, plist, pchunks, part_chunk_off,    \
									ready, err, spin))
	if (acc == 0 && bdata) {
		if (sparse)
			GDN_PARTS(0, true, true);
		else
			GDN_PARTS(0, true, false);
	} else if (acc == 1 && bdata) {
		if (sparse)
			GDN_PARTS(1, true, true);
		else
			GDN_PARTS(1, true, false);
	} else if (acc == 2 && !bdata) {
		if (sparse)
			GDN_PARTS(2, false, true);
		else
			GDN_PARTS(2, false, false);
	} else {
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "kinetic sweep: unsupported accumulate / boundary mode");
	}
#undef GDN_PARTS
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// CTAs of the spatial-parts sweep that fit on the device at once
template <typename F, typename Y, typename T>
int kin_parts_grid(int device, int acc, int sparse, int *grid)
{
	int nsm = 0, per = 0;
	GDN_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
	const void *fn;
	if (sparse)
		fn = acc == 0   ? (const void *)kin_parts_kernel<F, Y, T, 0, true, true>
			 : acc == 1 ? (const void *)kin_parts_kernel<F, Y, T, 1, true, true>
						: (const void *)kin_parts_kernel<F, Y, T, 2, false, true>;
	else
		fn = acc == 0   ? (const void *)kin_parts_kernel<F, Y, T, 0, true, false>
			 : acc == 1 ? (const void *)kin_parts_kernel<F, Y, T, 1, true, false>
						: (const void *)kin_parts_kernel<F, Y, T, 2, false, false>;
	GDN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kSwThreads, 0));
	*grid = nsm * (per > 0 ? per : 1);
	return GDN_CUDA_OK;
}

template <typename F, typename Y, typename T>
int launch_kin_sweep(const KinSweepParams &p, int acc, int bdata, int sparse, cudaStream_t s)
{
	const long long n = (long long)p.item_end - p.item_begin;
	if (n <= 0)
		return GDN_CUDA_OK;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)((n + kSwItems - 1) / kSwItems));
	cfg.blockDim = dim3(kSwThreads);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
#define GDN_SWEEP(A, B, SP) GDN_CUDA_TRY(cudaLaunchKernelEx(&cfg, kin_sweep_kernel<F, Y, T, A, B, SP>, p))
	if (acc == 0 && bdata) {
		if (sparse)
			GDN_SWEEP(0, true, true);
		else
			GDN_SWEEP(0, true, false);
	} else if (acc == 1 && bdata) {
		if (sparse)
			GDN_SWEEP(1, true, true);
		else
			GDN_SWEEP(1, true, false);
	} else if (acc == 2 && !bdata) {
		if (sparse)
			GDN_SWEEP(2, false, true);
		else
			GDN_SWEEP(2, false, false);
	} else {
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "kinetic sweep: unsupported accumulate / boundary mode");
	}
#undef GDN_SWEEP
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template <typename F, typename Y, typename T>
int launch_kin_levels(const KinSweepParams &p, const int *level_off, int nlevels, int grid, unsigned *bar, int *err,
					  long long spin, int acc, int bdata, int sparse, cudaStream_t s)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)grid);
	cfg.blockDim = dim3(kSwThreads);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	GDN_CUDA_TRY(cudaMemsetAsync(bar, 0, sizeof(unsigned), s));
#define GDN_LEVELS(A, B, SP)                                                                                          \
	GDN_CUDA_TRY(cudaLaunchKernelEx(&cfg, kin_levels_kernel<F, Y, T, A, B, SP>, p, level_off, nlevels, bar, err, spin))
	if (acc == 0 && bdata) {
		if (sparse)
			GDN_LEVELS(0, true, true);
		else
			GDN_LEVELS(0, true, false);
	} else if (acc == 1 && bdata) {
		if (sparse)
			GDN_LEVELS(1, true, true);
		else
			GDN_LEVELS(1, true, false);
	} else if (acc == 2 && !bdata) {
		if (sparse)
			GDN_LEVELS(2, false, true);
		else
			GDN_LEVELS(2, false, false);
	} else {
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "kinetic sweep: unsupported accumulate / boundary mode");
	}
#undef GDN_LEVELS
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template <typename F, typename Y, typename T>
int launch_kin_flags(const KinSweepParams &p, const int2 *chunks, int nchunks, int grid, unsigned *queue, int *ready,
					 long long nitems, int *err, long long spin, int acc, int bdata, int sparse, cudaStream_t s)
{
	if (nchunks <= 0)
		return GDN_CUDA_OK;
	GDN_CUDA_TRY(cudaMemsetAsync(ready, 0, (size_t)nitems * sizeof(int), s));
	GDN_CUDA_TRY(cudaMemsetAsync(queue, 0, sizeof(unsigned), s));
	const unsigned g = (unsigned)(grid < nchunks ? grid : nchunks);
#define GDN_FLAGS(A, B, SP)                                                                                           \
	kin_flags_kernel<F, Y, T, A, B, SP><<<g, kSwThreads, 0, s>>>(p, chunks, nchunks, queue, ready, err, spin)
	if (acc == 0 && bdata) {
		if (sparse)
			GDN_FLAGS(0, true, true);
		else
			GDN_FLAGS(0, true, false);
	} else if (acc == 1 && bdata) {
		if (sparse)
			GDN_FLAGS(1, true, true);
		else
			GDN_FLAGS(1, true, false);
	} else if (acc == 2 && !bdata) {
		if (sparse)
			GDN_FLAGS(2, false, true);
		else
			GDN_FLAGS(2, false, false);
	} else {
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "kinetic sweep: unsupported accumulate / boundary mode");
	}
#undef GDN_FLAGS
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// CTAs of the flag-driven sweep that fit on the device at once
template <typename F, typename Y, typename T>
int kin_flags_grid(int device, int acc, int sparse, int *grid)
{
	int nsm = 0, per = 0;
	GDN_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
	const void *fn;
	if (sparse)
		fn = acc == 0   ? (const void *)kin_flags_kernel<F, Y, T, 0, true, true>
			 : acc == 1 ? (const void *)kin_flags_kernel<F, Y, T, 1, true, true>
						: (const void *)kin_flags_kernel<F, Y, T, 2, false, true>;
	else
		fn = acc == 0   ? (const void *)kin_flags_kernel<F, Y, T, 0, true, false>
			 : acc == 1 ? (const void *)kin_flags_kernel<F, Y, T, 1, true, false>
						: (const void *)kin_flags_kernel<F, Y, T, 2, false, false>;
	GDN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kSwThreads, 0));
	// at most 4 CTAs per SM: the chunks in flight then poll and publish least
	// against each other (64^3 FP32 ms per step for 2 to 6 CTAs per SM: 5.20,
	// 4.56, 4.35, 4.46, 4.54)
	const int cap = 4;
	*grid = nsm * (per > cap ? cap : (per > 0 ? per : 1));
	return GDN_CUDA_OK;
}

// CTAs of the persistent level loop that fit on the device at once
template <typename F, typename Y, typename T>
int kin_levels_grid(int device, int acc, int sparse, int *grid)
{
	int nsm = 0, per = 0;
	GDN_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
	const void *fn;
	if (sparse)
		fn = acc == 0   ? (const void *)kin_levels_kernel<F, Y, T, 0, true, true>
			 : acc == 1 ? (const void *)kin_levels_kernel<F, Y, T, 1, true, true>
						: (const void *)kin_levels_kernel<F, Y, T, 2, false, true>;
	else
		fn = acc == 0   ? (const void *)kin_levels_kernel<F, Y, T, 0, true, false>
			 : acc == 1 ? (const void *)kin_levels_kernel<F, Y, T, 1, true, false>
						: (const void *)kin_levels_kernel<F, Y, T, 2, false, false>;
	GDN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kSwThreads, 0));
	// at most 3 CTAs per SM, about one per 32-item chunk of a 64^3 level: fewer
	// arrivals per grid barrier (64^3 FP32 ms per step for 2 / 3 / 4 CTAs per
	// SM: 6.04, 5.81, 6.75)
	*grid = nsm * (per > 3 ? 3 : per);
	return GDN_CUDA_OK;
}

#define GDN_LEVELS_INST(F, Y, T)                                                                                      \
	template int launch_kin_levels<F, Y, T>(const KinSweepParams &, const int *, int, int, unsigned *, int *,         \
											long long, int, int, int, cudaStream_t);                                     \
	template int kin_levels_grid<F, Y, T>(int, int, int, int *);                                                      \
	template int launch_kin_flags<F, Y, T>(const KinSweepParams &, const int2 *, int, int, unsigned *, int *,         \
										   long long, int *, long long, int, int, int, cudaStream_t);                    \
	template int kin_flags_grid<F, Y, T>(int, int, int, int *);                                                       \
	template int launch_kin_parts<F, Y, T>(const KinSweepParams &, const int *, const int2 *, const int *, int,       \
										   int *, long long, int *, long long, int, int, int, cudaStream_t);             \
	template int kin_parts_grid<F, Y, T>(int, int, int, int *);
GDN_LEVELS_INST(double, double, double)
GDN_LEVELS_INST(float, float, float)
GDN_LEVELS_INST(__nv_bfloat16, float, float)
GDN_LEVELS_INST(double, float, float)
#undef GDN_LEVELS_INST

template int launch_kin_sweep<double, double, double>(const KinSweepParams &, int, int, int, cudaStream_t);
template int launch_kin_sweep<float, float, float>(const KinSweepParams &, int, int, int, cudaStream_t);
template int launch_kin_sweep<__nv_bfloat16, float, float>(const KinSweepParams &, int, int, int, cudaStream_t);
template int launch_kin_sweep<double, float, float>(const KinSweepParams &, int, int, int, cudaStream_t);

// FP64 residual of the transport system of every item (no level order: it
// only reads y), same thread layout as the sweep:
//   r = f - y - coef Minv (V y + sum_outflow s E S E^T y + sum_inflow s E S tr)
// with V_ij = -(u . D_ij), u_k = v . codtau[:, k], tr the upwind neighbour's
// y or the boundary f_eq.  This is f - b - M1 y with M1 as the blocks kernel
// builds it, from the FP64 u, theta dt / det and v.vn it records per item.
template <bool SPARSE>
__global__ void __launch_bounds__(kSwThreads) kin_residual_kernel(KinResidualParams p)
{
	const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
	const long long k = (long long)blockIdx.x * kSwItems + lane;
	if (k >= p.nitems)
		return;
	const Tables<double> &tb = c_tab_d;
	const int4 nb4 = p.rnb[k];
	const int4 pm4 = p.rpm[k];
	const int nbk[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
	const int pmk[4] = {pm4.x, pm4.y, pm4.z, pm4.w};
	double tr[4][6];
#pragma unroll
	for (int f = 0; f < 4; f++) {
		const int nbv = nbk[f];
		if (nbv >= 0) {
			const double *yn = p.yacc + (long long)nbv * 60 + c * 10;
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				tr[f][jj] = yn[(pmk[f] >> (4 * jj)) & 15];
		} else if (nbv != INT_MIN) {
			const int v = p.items[k] % p.nv;
			const double *b = p.bt + (((long long)(-nbv - 1) * p.nv + v) * 6 + c) * 6;
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				tr[f][jj] = b[jj];
		} else {
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				tr[f][jj] = 0.0;
		}
	}
	double yk[10], fv[10];
	load10<double, double>(p.yacc + k * 60 + c * 10, yk);
	load10<double, double>(p.f + k * 60 + c * 10, fv);
	const double4 ru = p.ru64[k]; // u_0, u_1, u_2, theta dt / det
	const double4 s4 = p.rs64[k];
	const double s[4] = {s4.x, s4.y, s4.z, s4.w};
	// V y = -(u_0 D_0 y + u_1 D_1 y + u_2 D_2 y)
	double t[10];
#pragma unroll
	for (int i = 0; i < 10; i++) {
		double g[3];
#pragma unroll
		for (int q = 0; q < 3; q++) {
			double acc = 0.0;
#pragma unroll
			for (int j = 0; j < 10; j++)
				if (!SPARSE || (dmask(q, i) >> j & 1))
					acc += tb.D[q][i][j] * yk[j];
			g[q] = acc;
		}
		t[i] = -(ru.x * g[0] + ru.y * g[1] + ru.z * g[2]);
	}
#pragma unroll
	for (int f = 0; f < 4; f++) {
		const bool out = s[f] > 0.0;
#pragma unroll
		for (int ii = 0; ii < 6; ii++) {
			double acc = 0.0;
#pragma unroll
			for (int jj = 0; jj < 6; jj++)
				if (!SPARSE || (smask(ii) >> jj & 1))
					acc += tb.S[ii][jj] * (out ? yk[f2n(f, jj)] : tr[f][jj]);
			t[f2n(f, ii)] += acc * s[f];
		}
	}
	float rr[10];
#pragma unroll
	for (int i = 0; i < 10; i++) {
		double acc = 0.0;
#pragma unroll
		for (int j = 0; j < 10; j++)
			acc += tb.Minv[i][j] * t[j];
		rr[i] = (float)(fv[i] - yk[i] - ru.w * acc);
	}
	store10<float, float>(p.r + k * 60 + c * 10, rr);
}

int launch_kin_residual(const KinResidualParams &p, int sparse, cudaStream_t s)
{
	if (p.nitems <= 0)
		return GDN_CUDA_OK;
	const unsigned grid = (unsigned)((p.nitems + kSwItems - 1) / kSwItems);
	if (sparse)
		kin_residual_kernel<true><<<grid, kSwThreads, 0, s>>>(p);
	else
		kin_residual_kernel<false><<<grid, kSwThreads, 0, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// x = a_y y + a_f f (the Crank-Nicolson transport result), then the
// relaxation of dg_apply_relaxation (dg.c:109-147): w = sum_v x_v,
// f <- omega f_eq(w) + (1 - omega) x.  A thread per (element, node).
template <typename F, typename Y, typename T, int NV>
__global__ void kin_relax_kernel(KinRelaxParams p)
{
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (t >= p.ne * 10)
		return;
	const long long e = t / 10;
	const int i = (int)(t % 10);
	F *f = reinterpret_cast<F *>(p.f);
	const Y *yv = reinterpret_cast<const Y *>(p.y);
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
			const T xv = (T)p.a_y * (T)Store<Y>::load(yv + o) + (T)p.a_f * (T)Store<F>::load(f + o);
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
			Store<F>::store(f + base[v] + c * 10, om * feq + om1 * x[v][c]);
		}
	}
}

template <typename F, typename Y, typename T>
int launch_kin_relax(const KinRelaxParams &p, cudaStream_t s)
{
	const unsigned nblk = (unsigned)((p.ne * 10 + 255) / 256);
	if (p.nv == 4)
		kin_relax_kernel<F, Y, T, 4><<<nblk, 256, 0, s>>>(p);
	else
		kin_relax_kernel<F, Y, T, 6><<<nblk, 256, 0, s>>>(p);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_relax<double, double, double>(const KinRelaxParams &, cudaStream_t);
template int launch_kin_relax<float, float, float>(const KinRelaxParams &, cudaStream_t);
template int launch_kin_relax<__nv_bfloat16, float, float>(const KinRelaxParams &, cudaStream_t);

} // namespace gdn
