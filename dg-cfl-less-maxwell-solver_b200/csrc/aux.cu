// Setup and support kernels: FP64 geometry (K0), initial data, boundary dofs,
// layout conversion between the reference's wn and the device layouts, and
// the deterministic FP64 L2 error norm (K2).
#include "aux.h"

namespace gdn {

// K0: per element codtau (row-major) and det, FP64 in the reference's order
// (gdn_tetra_ref2phy + mesh_get_elem_det), from the vertex P2 nodes.
__global__ void geometry_kernel(const int *__restrict__ e2q, const double *__restrict__ node, long long ne,
								double *__restrict__ geom, int *__restrict__ bad)
{
	const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (e >= ne)
		return;
	double p[4][3], dtau[3][3], cod[3][3], det;
	for (int v = 0; v < 4; v++) {
		const long long q = e2q[e * 10 + v];
		for (int c = 0; c < 3; c++)
			p[v][c] = node[3 * q + c];
	}
	gdn_geometry_from_vertices(p, dtau, cod, &det);
	for (int a = 0; a < 3; a++)
		for (int b = 0; b < 3; b++)
			geom[e * 10 + 3 * a + b] = cod[a][b];
	geom[e * 10 + 9] = det;
	if (!(det > 0.0))
		atomicMax(bad, 1);
}

int launch_geometry(const int *e2q, const double *node, long long ne, double *geom, int *bad, cudaStream_t s)
{
	geometry_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(e2q, node, ne, geom, bad);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

template <typename T>
__global__ void convert_kernel(const double *__restrict__ a, T *__restrict__ b, long long n)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i < n)
		b[i] = (T)a[i];
}

template <typename T>
int launch_convert(const double *a, T *b, long long n, cudaStream_t s)
{
	if (n <= 0)
		return GDN_CUDA_OK;
	convert_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_convert<float>(const double *, float *, long long, cudaStream_t);
template int launch_convert<__nv_bfloat16>(const double *, __nv_bfloat16 *, long long, cudaStream_t);

__global__ void widen_kernel_f(const float *__restrict__ a, double *__restrict__ b, long long n)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i < n)
		b[i] = (double)a[i];
}

int launch_widen(const float *a, double *b, long long n, cudaStream_t s)
{
	if (n <= 0)
		return GDN_CUDA_OK;
	widen_kernel_f<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

__device__ __forceinline__ void node_xyz(const int *e2q, const double *node, long long e, int i, double x[3])
{
	const long long q = e2q[e * 10 + i];
	x[0] = node[3 * q + 0];
	x[1] = node[3 * q + 1];
	x[2] = node[3 * q + 2];
}

// dg_init_sol_macro, RK3 branch (src/dg/dg.c:32-59): w = w_exact(x, 0) for
// the elements e0 .. e0 + ne - 1 (e2q points at element e0), tiled layout
template <typename S>
__global__ void init_rk3_kernel(const int *__restrict__ e2q, const double *__restrict__ node, long long ne,
								long long e0, Data d, S *__restrict__ w)
{
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (t >= ne * 10)
		return;
	const long long e = t / 10;
	const int i = (int)(t % 10);
	double x[3], we[6];
	node_xyz(e2q, node, e, i, x);
	exact_w(d, x, 0.0, we);
	for (int c = 0; c < 6; c++)
		Store<S>::store(w + rk3_tix(e0 + e, i * 6 + c), we[c]);
}

template <typename S>
int launch_init_rk3(const int *e2q, const double *node, long long ne, long long e0, const Data &d, S *w,
					cudaStream_t s)
{
	init_rk3_kernel<S><<<(unsigned)((ne * 10 + 255) / 256), 256, 0, s>>>(e2q, node, ne, e0, d, w);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_init_rk3<double>(const int *, const double *, long long, long long, const Data &, double *,
									 cudaStream_t);
template int launch_init_rk3<float>(const int *, const double *, long long, long long, const Data &, float *,
									cudaStream_t);

// f_eq of the kinetic model: f_v = w / nv + feq_c A(v) w
__device__ __forceinline__ void feq_component(const double w[6], const double *v, int nv, double feq_c,
											  double out[6])
{
	double n[3] = {v[0], v[1], v[2]}, Aw[6];
	maxwell_A<double>(n, w, Aw);
	for (int c = 0; c < 6; c++)
		out[c] = w[c] / nv + feq_c * Aw[c];
}

// dg_init_sol_macro, kinetic branch: f = f_eq(w_exact(x, 0)); layout
// f[k][c][i] with k = pos[e * nv + v] (sweep order)
template <typename S>
__global__ void init_kin_kernel(const int *__restrict__ e2q, const double *__restrict__ node, long long ne,
								Data d, KinModel km, const int *__restrict__ pos, S *__restrict__ f)
{
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (t >= ne * 10)
		return;
	const long long e = t / 10;
	const int i = (int)(t % 10);
	double x[3], we[6], fe[6];
	node_xyz(e2q, node, e, i, x);
	exact_w(d, x, 0.0, we);
	for (int v = 0; v < km.nv; v++) {
		feq_component(we, km.vi + 3 * v, km.nv, km.feq_c, fe);
		for (int c = 0; c < 6; c++)
			Store<S>::store(f + ((long long)pos[e * km.nv + v] * 6 + c) * 10 + i, fe[c]);
	}
}

template <typename S>
int launch_init_kin(const int *e2q, const double *node, long long ne, const Data &d, const KinModel &km,
					const int *pos, S *f, cudaStream_t s)
{
	init_kin_kernel<S><<<(unsigned)((ne * 10 + 255) / 256), 256, 0, s>>>(e2q, node, ne, d, km, pos, f);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_init_kin<double>(const int *, const double *, long long, const Data &, const KinModel &,
									 const int *, double *, cudaStream_t);
template int launch_init_kin<float>(const int *, const double *, long long, const Data &, const KinModel &,
									const int *, float *, cudaStream_t);
template int launch_init_kin<__nv_bfloat16>(const int *, const double *, long long, const Data &,
											const KinModel &, const int *, __nv_bfloat16 *, cudaStream_t);

// Boundary dofs of the reference layout.  RK3: w_exact(x_L, t)
// (dg_update_boundary, dg.c:101-104); kinetic: f_eq(w_exact(x_L, t))
// (d3q4_get_fR with use_feq, d3q4.c:289-301).  out points at the first
// boundary dof; RK3 stride: [(bf*6 + jj)*6 + c]; kinetic: [(c*nv + v)*neq + ..].
__global__ void boundary_dofs_kernel(const double *__restrict__ bxyz, long long nbf, Data d, double t, int kinetic,
									 KinModel km, long long neq, double *__restrict__ out)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= nbf * 6)
		return;
	double x[3] = {bxyz[3 * u], bxyz[3 * u + 1], bxyz[3 * u + 2]}, we[6];
	exact_w(d, x, t, we);
	if (!kinetic) {
		for (int c = 0; c < 6; c++)
			out[u * 6 + c] = we[c];
	} else {
		double fe[6];
		for (int v = 0; v < km.nv; v++) {
			feq_component(we, km.vi + 3 * v, km.nv, km.feq_c, fe);
			for (int c = 0; c < 6; c++)
				out[(long long)(c * km.nv + v) * neq + u] = fe[c];
		}
	}
}

// RK3 boundary traces at a stage time, in the stage kernels' precision:
// out[(bf*6 + jj)*6 + c] = w_exact(x_{bf,jj}, t)_c  (dg_update_boundary,
// dg.c:101-104, evaluated once per stage instead of inside the flux loop),
// with the data, time and time step of the face's instance.  The stage time
// t + C_i dt is formed from the device copy of t with the host's rounding (no
// fused multiply-add), so every stage sees the reference's time bits.
template <typename T>
__global__ void boundary_trace_kernel(const double *__restrict__ bxyz, long long nbf, Batch b, double c_stage,
									  T *__restrict__ out)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= nbf * 6)
		return;
	const int inst = b.bfinst ? b.bfinst[u / 6] : 0;
	const double t = __dadd_rn(b.t[inst], __dmul_rn(c_stage, b.dt[inst]));
	double x[3] = {bxyz[3 * u], bxyz[3 * u + 1], bxyz[3 * u + 2]}, we[6];
	exact_w(b.data[inst], x, t, we);
	for (int c = 0; c < 6; c++)
		out[u * 6 + c] = (T)we[c];
}

template <typename T>
int launch_boundary_trace(const double *bxyz, long long nbf, const Batch &b, double c_stage, T *out, cudaStream_t s)
{
	if (nbf <= 0)
		return GDN_CUDA_OK;
	boundary_trace_kernel<T><<<(unsigned)((nbf * 6 + 255) / 256), 256, 0, s>>>(bxyz, nbf, b, c_stage, out);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_boundary_trace<double>(const double *, long long, const Batch &, double, double *, cudaStream_t);
template int launch_boundary_trace<float>(const double *, long long, const Batch &, double, float *, cudaStream_t);

// device time of every instance: t = value, and t += dt (the reference's
// accumulation, explicit.c:103 / relaxation.c:171)
__global__ void set_time_kernel(Batch b, double value)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < b.ninst)
		b.t[i] = value;
}
__global__ void advance_time_kernel(Batch b)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < b.ninst)
		b.t[i] = __dadd_rn(b.t[i], b.dt[i]);
}
int launch_set_time(const Batch &b, double value, cudaStream_t s)
{
	set_time_kernel<<<(b.ninst + 127) / 128, 128, 0, s>>>(b, value);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
int launch_advance_time(const Batch &b, cudaStream_t s)
{
	advance_time_kernel<<<(b.ninst + 127) / 128, 128, 0, s>>>(b);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

int launch_boundary_dofs(const double *bxyz, long long nbf, const Data &d, double t, int kinetic,
						 const KinModel &km, long long neq, double *out, cudaStream_t s)
{
	if (nbf <= 0)
		return GDN_CUDA_OK;
	boundary_dofs_kernel<<<(unsigned)((nbf * 6 + 255) / 256), 256, 0, s>>>(bxyz, nbf, d, t, kinetic, km, neq,
																		   out);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// the analytic data at arbitrary points: w[i][c] = w_exact(xyz[i], t)_c
__global__ void eval_data_kernel(const double *__restrict__ xyz, long long n, Data d, double t,
								 double *__restrict__ w)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= n)
		return;
	double x[3] = {xyz[3 * u], xyz[3 * u + 1], xyz[3 * u + 2]}, we[6];
	exact_w(d, x, t, we);
	for (int c = 0; c < 6; c++)
		w[u * 6 + c] = we[c];
}

int launch_eval_data(const double *xyz, long long n, const Data &d, double t, double *w, cudaStream_t s)
{
	if (n <= 0)
		return GDN_CUDA_OK;
	eval_data_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(xyz, n, d, t, w);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

// kinetic device layout f[k][c][i], k = pos[e * nv + v]
//   <->  wn[(c*nv + v)*neq + 10 e + i]
template <typename S>
__global__ void kin_pack_kernel(const S *__restrict__ f, const int *__restrict__ pos, long long ne, int nv,
								long long neq, double *__restrict__ wn, int to_ref)
{
	const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	const long long tot = ne * nv * 60;
	if (t >= tot)
		return;
	const int i = (int)(t % 10);
	const int c = (int)((t / 10) % 6);
	const long long ev = t / 60;
	const int v = (int)(ev % nv);
	const long long e = ev / nv;
	const long long r = (long long)(c * nv + v) * neq + e * 10 + i;
	const long long o = (long long)pos[ev] * 60 + c * 10 + i;
	if (to_ref)
		wn[r] = (double)Store<S>::load(f + o);
	else
		Store<S>::store(const_cast<S *>(f) + o, wn[r]);
}

template <typename S>
int launch_kin_pack(const S *f, const int *pos, long long ne, int nv, long long neq, double *wn, int to_ref,
					cudaStream_t s)
{
	const long long tot = ne * nv * 60;
	kin_pack_kernel<S><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(f, pos, ne, nv, neq, wn, to_ref);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_kin_pack<double>(const double *, const int *, long long, int, long long, double *, int,
									 cudaStream_t);
template int launch_kin_pack<float>(const float *, const int *, long long, int, long long, double *, int,
									cudaStream_t);
template int launch_kin_pack<__nv_bfloat16>(const __nv_bfloat16 *, const int *, long long, int, long long, double *,
											int, cudaStream_t);

// K2: simulation_error_l2 (src/simulation/simulation.c:606-666).  Pass 1: one
// FP64 partial per block and field, in a fixed order; pass 2: one block sums
// the partials in order.  Deterministic for a given launch shape.
template <typename S>
__global__ void error_partial_kernel(const S *__restrict__ state, int kinetic, long long e0, int nv,
									 const int *__restrict__ pos,
									 const int *__restrict__ e2q, const double *__restrict__ node,
									 const double *__restrict__ geom, long long ne, Data d, double t,
									 double *__restrict__ partial)
{
	__shared__ double red[6][256];
	double acc[6] = {0, 0, 0, 0, 0, 0};
	const Tables<double> &tb = c_tab_d;
	for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < ne * 10;
		 u += (long long)gridDim.x * blockDim.x) {
		const long long e = u / 10;
		const int i = (int)(u % 10);
		double x[3], we[6], wl[6];
		node_xyz(e2q, node, e, i, x);
		exact_w(d, x, t, we);
		if (!kinetic) {
			for (int c = 0; c < 6; c++)
				wl[c] = (double)Store<S>::load(state + rk3_tix(e0 + e, i * 6 + c));
		} else {
			for (int c = 0; c < 6; c++) {
				double s = 0.0;
				for (int v = 0; v < nv; v++)
					s += (double)Store<S>::load(state + ((long long)pos[e * nv + v] * 6 + c) * 10 + i);
				wl[c] = s;
			}
		}
		const double det = geom[e * 10 + 9];
		for (int c = 0; c < 6; c++) {
			const double diff = wl[c] - we[c];
			acc[c] += diff * diff * tb.wpg[i] * det;
		}
	}
	for (int c = 0; c < 6; c++)
		red[c][threadIdx.x] = acc[c];
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if ((int)threadIdx.x < w)
			for (int c = 0; c < 6; c++)
				red[c][threadIdx.x] += red[c][threadIdx.x + w];
		__syncthreads();
	}
	if (threadIdx.x == 0)
		for (int c = 0; c < 6; c++)
			partial[blockIdx.x * 6 + c] = red[c][0];
}

__global__ void error_final_kernel(const double *__restrict__ partial, int nblk, double *__restrict__ out)
{
	__shared__ double red[6][256];
	double acc[6] = {0, 0, 0, 0, 0, 0};
	for (int b = threadIdx.x; b < nblk; b += blockDim.x)
		for (int c = 0; c < 6; c++)
			acc[c] += partial[b * 6 + c];
	for (int c = 0; c < 6; c++)
		red[c][threadIdx.x] = acc[c];
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if ((int)threadIdx.x < w)
			for (int c = 0; c < 6; c++)
				red[c][threadIdx.x] += red[c][threadIdx.x + w];
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		double e = 0.0;
		for (int c = 0; c < 6; c++) {
			out[1 + c] = red[c][0];
			e += sqrt(fabs(red[c][0])) / 6.0;
		}
		out[0] = e;
	}
}

template <typename S>
int launch_error_l2(const S *state, int kinetic, long long e0, int nv, const int *pos, const int *e2q,
					const double *node, const double *geom, long long ne, const Data &d, double t, double *partial,
					int nblk, double *out, cudaStream_t s)
{
	error_partial_kernel<S><<<nblk, 256, 0, s>>>(state, kinetic, e0, nv, pos, e2q, node, geom, ne, d, t, partial);
	GDN_CUDA_TRY(cudaGetLastError());
	error_final_kernel<<<1, 256, 0, s>>>(partial, nblk, out);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}
template int launch_error_l2<double>(const double *, int, long long, int, const int *, const int *, const double *,
									 const double *, long long, const Data &, double, double *, int, double *,
									 cudaStream_t);
template int launch_error_l2<float>(const float *, int, long long, int, const int *, const int *, const double *,
									const double *, long long, const Data &, double, double *, int, double *,
									cudaStream_t);
template int launch_error_l2<__nv_bfloat16>(const __nv_bfloat16 *, int, long long, int, const int *, const int *,
											const double *, const double *, long long, const Data &, double, double *,
											int, double *, cudaStream_t);

// Nodal values for output (io_hdf5.c:179-213): each P2 node of instance
// elements [e0, e0 + ne) takes its dofs from the first element containing it
// and the first local node there (node2elem is filled in element order,
// mesh.c:1208-1221): the smallest 10 e + iloc.
__global__ void io_owner_kernel(const int *__restrict__ e2q, long long e0, long long ne, long long q0, int *owner)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= ne * 10)
		return;
	atomicMin(owner + (e2q[10 * e0 + u] - q0), (int)u);
}

template <typename S>
__global__ void io_values_kernel(const S *__restrict__ st, int kinetic, int nv, const int *__restrict__ pos,
								 long long e0, long long nq, const int *__restrict__ owner, double *__restrict__ out)
{
	const long long in = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (in >= nq)
		return;
	const int u = owner[in];
	if (u == 0x7f7f7f7f) { // a node no element uses (the fill value)
		for (int im = 0; im < (kinetic ? 6 * nv : 6); im++)
			out[im * nq + in] = 0.0;
		return;
	}
	const long long e = e0 + u / 10;
	const int i = u % 10;
	if (!kinetic) {
		for (int c = 0; c < 6; c++)
			out[c * nq + in] = (double)Store<S>::load(st + rk3_tix(e, i * 6 + c));
	} else {
		// component im = iw * nv + iv of the reference's kinetic wn
		for (int v = 0; v < nv; v++) {
			const long long k = pos[e * nv + v];
			for (int c = 0; c < 6; c++)
				out[(c * nv + v) * nq + in] = (double)Store<S>::load(st + k * 60 + c * 10 + i);
		}
	}
}

int launch_node_values(const void *st, int sk, int kinetic, int nv, const int *pos, const int *e2q, long long e0,
					   long long ne, long long q0, long long nq, int *owner, double *out, cudaStream_t s)
{
	if (nq <= 0)
		return GDN_CUDA_OK;
	GDN_CUDA_TRY(cudaMemsetAsync(owner, 0x7f, nq * sizeof(int), s)); // 0x7f7f7f7f: above every 10 e + i
	io_owner_kernel<<<(unsigned)((ne * 10 + 255) / 256), 256, 0, s>>>(e2q, e0, ne, q0, owner);
	GDN_CUDA_TRY(cudaGetLastError());
	const unsigned g = (unsigned)((nq + 255) / 256);
	if (sk == 0)
		io_values_kernel<double><<<g, 256, 0, s>>>(reinterpret_cast<const double *>(st), kinetic, nv, pos, e0, nq,
												   owner, out);
	else if (sk == 1)
		io_values_kernel<float><<<g, 256, 0, s>>>(reinterpret_cast<const float *>(st), kinetic, nv, pos, e0, nq,
												  owner, out);
	else
		io_values_kernel<__nv_bfloat16><<<g, 256, 0, s>>>(reinterpret_cast<const __nv_bfloat16 *>(st), kinetic, nv,
														   pos, e0, nq, owner, out);
	GDN_CUDA_TRY(cudaGetLastError());
	return GDN_CUDA_OK;
}

} // namespace gdn
