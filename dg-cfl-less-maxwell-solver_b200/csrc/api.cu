// The C-ABI of include/gdon3d_cuda.h: handle life cycle, attach (setup on the
// device), the time loops, state conversion and norms.  Host orchestration
// only; the arithmetic is in rk3.cu, kinetic.cu and aux.cu.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "aux.h"
#include "kernels.h"

namespace gdn {
template <typename GT>
int launch_kin_setup(const int *face2elem, long long nf, const double *geom, const int *nb, long long ne,
					 const KinModel &km, double *sown64, unsigned char *mask, cudaStream_t s);
int kin_upload_block_tables(const gdn_cuda_tables *t);
template <typename GT>
int launch_kin_blocks(const double *geom, const double *sown64, const int *items, const int *pos, const int *nb,
					  const int *perm, long long ne, const KinModel &km, double theta, const int *einst,
					  const double *dt_tab, GT *G, GT *rcoef, int4 *rnb, int4 *rpm, GT *rs, double4 *ru64,
					  double4 *rs64, int *bad, cudaStream_t s);
}

using namespace gdn;

// ---------------------------------------------------------------- errors --
static thread_local std::string g_last_error;

int gdn_set_error(int code, const char *msg)
{
	g_last_error = msg ? msg : "";
	return code;
}

int gdn_cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
	char buf[512];
	std::snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what,
				  file, line);
	g_last_error = buf;
	return e == cudaErrorMemoryAllocation ? GDN_CUDA_ERR_OOM : GDN_CUDA_ERR_CUDA;
}

extern "C" const char *gdn_cuda_last_error(void)
{
	return g_last_error.c_str();
}

#define GDN_TRY(expr)                                                                              \
	do {                                                                                           \
		int _rc = (expr);                                                                          \
		if (_rc != GDN_CUDA_OK)                                                                    \
			return _rc;                                                                            \
	} while (0)

// ---------------------------------------------------------------- handle --
struct DevBuf {
	void *p = nullptr;
	size_t bytes = 0;
};

struct gdn_cuda_handle {
	int device = 0;
	cudaStream_t stream = nullptr;
	int scheme = 0, precision = 0, nv = 0, use_graph = 1;
	long long ne = 0, nf = 0, nbf = 0, nq = 0, neq = 0;
	double theta = 0.5, omega = 0, lambda = 0;
	KinModel km{};
	long long steps = 0;
	long long launches = 0;
	int ssize = 8; // bytes per stored state value
	int rk3_sparse = 1; // tables follow the P2 structural-zero pattern
	int rk3_fact = 1; // and the derivative tables factor through the P1 basis
	int num_sms = 148; // SMs of the device
	int bc_metal = 0; // RK3 boundary faces take the metal flux
	// device arrays
	std::vector<DevBuf> bufs;
	int *e2q = nullptr;
	double *node = nullptr;
	double *geom64 = nullptr;
	void *geomT = nullptr;
	int *nb = nullptr;
	int *perm = nullptr;
	int *face2elem = nullptr;
	double *bxyz = nullptr;
	double *partial = nullptr;
	double *result = nullptr; // [7]
	double *staging = nullptr; // m * neq doubles (reference layout)
	int *flag = nullptr;
	double *host_result = nullptr; // pinned [8]
	int nblk_err = 0;
	// RK3
	void *w[2] = {nullptr, nullptr};
	void *k2 = nullptr;
	void *btrace = nullptr; // [nbf][6][6] boundary traces at the stage time
	int cur = 0;
	int rk3_variant = 0; // stage kernel for fewer (0) / more (1) resident CTAs per SM
	bool rk3_autotune = true; // pick the variant at attach by timing both
	// kinetic, in sweep order (item k = position in the level-sorted list)
	// f: FP64 (FP64, FP32_REFINE), FP32 or BF16; y: FP64 or FP32; G, rs,
	// rcoef: FP64 (FP64) or FP32
	void *f = nullptr, *y = nullptr, *G = nullptr, *rcoef = nullptr;
	void *rs = nullptr; // [k][4] own-side v.vn
	int4 *rnb = nullptr, *rpm = nullptr; // [k] inflow neighbour items, permutations
	double *bt = nullptr; // [bf][v][6][6] boundary f_eq at t + dt/2
	double *sown64 = nullptr; // [e * nv + v][4] v.vn in FP64
	double4 *ru64 = nullptr, *rs64 = nullptr; // FP32_REFINE: [k] (u, theta dt / det), v.vn in FP64
	double *yacc = nullptr; // FP32_REFINE: FP64 solution of the transport solve
	float *rhs = nullptr; // FP32_REFINE: residual, right-hand side of the corrections
	int refine_passes = 1;
	int kin_mode = 1; // 1: a launch per sweep level, 2: one cooperative launch per sweep, 3: flag-driven,
	                  // 4: spatial parts
	bool kin_autotune = true; // pick kin_mode at attach by timing the modes
	int kin_grid[3] = {0, 0, 0}; // CTAs of the cooperative sweep, per accumulate mode
	int kin_fgrid[3] = {0, 0, 0}; // CTAs of the flag-driven sweep, per accumulate mode
	int2 *kchunks = nullptr; // [nchunks] level-aligned 32-item chunks (first item, end item)
	int nchunks = 0;
	int *kready = nullptr; // [nitems] readiness flags of the flag-driven sweep
	unsigned *kqueue = nullptr; // its chunk counter
	long long spin_limit = 1LL << 21; // polls of a bounded device-side wait (~1 s)
	// the spatial-parts sweep: item list by part, level-aligned chunks, chunk ranges per part
	int *plist = nullptr;
	int2 *pchunks = nullptr;
	int *part_chunk_off = nullptr;
	int nparts = 0;
	int kin_pgrid[3] = {0, 0, 0}; // CTAs of the parts sweep that fit at once, per accumulate mode
	int max_chunks = 1; // most 32-item chunks in one level
	int *level_off_dev = nullptr;
	unsigned *bar = nullptr; // [2] grid barrier of the cooperative sweep
	int *err = nullptr; // set on the device when a barrier wait gave up
	int *items = nullptr; // [k] e * nv + v
	int *pos = nullptr; // [e * nv + v] k
	std::vector<int> level_off;
	// device time and captured step loops
	double *t_dev = nullptr; // [ninst]
	cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
	long long graph_nodes[2] = {0, 0};
	// batch of instances: concatenated meshes, per-instance dt / data / time.
	// Offsets of instance i: elements e_off[i], boundary faces bf_off[i],
	// reference-layout state w_off[i] (m * neq_i values each).
	int ninst = 1;
	std::vector<long long> e_off, bf_off, w_off, neq_i, q_off;
	std::vector<Data> hdata;
	std::vector<double> hdt, ht, ht_bdof; // host mirrors of dt, t, RK3 boundary-data time
	int *einst = nullptr, *bfinst = nullptr; // nullptr for a single instance
	Data *data_dev = nullptr;
	double *dt_dev = nullptr;

	Batch batch() const
	{
		Batch b;
		b.einst = einst;
		b.bfinst = bfinst;
		b.data = data_dev;
		b.dt = dt_dev;
		b.t = t_dev;
		b.ninst = ninst;
		return b;
	}
};

template <typename X>
static int dalloc(gdn_cuda_handle *h, X **p, size_t count)
{
	void *q = nullptr;
	const size_t bytes = count * sizeof(X) > 0 ? count * sizeof(X) : 16;
	cudaError_t e = cudaMalloc(&q, bytes);
	if (e != cudaSuccess) {
		cudaGetLastError();
		char buf[160];
		std::snprintf(buf, sizeof(buf), "device allocation of %zu bytes failed", bytes);
		return gdn_set_error(GDN_CUDA_ERR_OOM, buf);
	}
	DevBuf b;
	b.p = q;
	b.bytes = bytes;
	h->bufs.push_back(b);
	*p = reinterpret_cast<X *>(q);
	return GDN_CUDA_OK;
}

static void free_handle(gdn_cuda_handle *h)
{
	if (!h)
		return;
	cudaSetDevice(h->device);
	if (h->stream)
		cudaStreamSynchronize(h->stream);
	for (int k = 0; k < 2; k++)
		if (h->graph_exec[k])
			cudaGraphExecDestroy(h->graph_exec[k]);
	for (auto &b : h->bufs)
		cudaFree(b.p);
	if (h->host_result)
		cudaFreeHost(h->host_result);
	if (h->stream)
		cudaStreamDestroy(h->stream);
	delete h;
}

// -------------------------------------------------------- table upload --
template <typename T>
static void fill_tables(const gdn_cuda_tables *t, Tables<T> &o)
{
	std::memset(&o, 0, sizeof(o));
	for (int k = 0; k < 3; k++)
		for (int i = 0; i < 10; i++)
			for (int j = 0; j < 10; j++)
				o.D[k][i][j] = (T)t->internal[i][j][k];
	for (int i = 0; i < 10; i++) {
		o.wpg[i] = (T)t->wpg[i];
		for (int j = 0; j < 10; j++) {
			o.Minv[i][j] = (T)t->inv_mass[i][j];
			o.M[i][j] = (T)t->mass[i][j];
		}
	}
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++)
			o.S[i][j] = (T)t->face_scal[i][j];
	for (int m = 0; m < 5; m++)
		for (int j = 0; j < 10; j++) {
			o.MinvP[m][j].x = o.Minv[2 * m][j];
			o.MinvP[m][j].y = o.Minv[2 * m + 1][j];
		}
	double q4[4][10];
	rk3_q4(t, q4);
	for (int l = 0; l < 4; l++)
		for (int j = 0; j < 10; j++)
			o.Q4[l][j] = (T)q4[l][j];
	double qs[6], ms[7], ss[5];
	rk3_sym_coeffs(t, qs, ms, ss);
	for (int k = 0; k < 5; k++)
		o.s_sym[k] = (T)ss[k];
	for (int k = 0; k < 6; k++)
		o.q4_sym[k] = (T)qs[k];
	for (int k = 0; k < 7; k++)
		o.minv_sym[k] = (T)ms[k];
	o.n3scale = (T)(t->ref_normal[3][0] * std::sqrt(3.0));
	for (int f = 0; f < 4; f++) {
		for (int k = 0; k < 3; k++)
			o.ref_normal[f][k] = t->ref_normal[f][k];
		for (int j = 0; j < 6; j++)
			o.f2n[f][j] = t->face2node[f][j];
	}
	for (int i = 0; i < 10; i++)
		o.nface_of_node[i] = 0;
	for (int f = 0; f < 4; f++)
		for (int j = 0; j < 6; j++) {
			const int i = t->face2node[f][j];
			const int a = o.nface_of_node[i]++;
			if (a < 3) {
				o.face_of_node[i][a] = f;
				o.pos_of_node[i][a] = j;
			}
		}
}

static int upload_tables(const gdn_cuda_tables *t)
{
	for (int f = 0; f < 4; f++)
		for (int j = 0; j < 6; j++)
			if (t->face2node[f][j] < 0 || t->face2node[f][j] > 9)
				return gdn_set_error(GDN_CUDA_ERR_INVALID, "tables: face2node out of range");
	Tables<double> td;
	Tables<float> tf;
	fill_tables(t, td);
	fill_tables(t, tf);
	for (int i = 0; i < 10; i++)
		if (td.nface_of_node[i] < 2 || td.nface_of_node[i] > 3)
			return gdn_set_error(GDN_CUDA_ERR_INVALID, "tables: face2node does not cover the P2 nodes");
	GDN_CUDA_TRY(cudaMemcpyToSymbol(c_tab_d, &td, sizeof(td)));
	GDN_CUDA_TRY(cudaMemcpyToSymbol(c_tab_f, &tf, sizeof(tf)));
	return GDN_CUDA_OK;
}

// ------------------------------------------------------------ attach --
static int validate_mesh(const gdn_cuda_mesh *m)
{
	if (!m || m->nbelems <= 0 || m->nbfaces <= 0 || m->nboundaryfaces < 0 || m->nbqnodes <= 0 ||
		!m->face2elem || !m->fnode2enode || !m->elem2qnode || !m->node ||
		(m->nboundaryfaces > 0 && !m->boundaryface))
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: mesh arrays or sizes missing");
	const long long ne = m->nbelems, nf = m->nbfaces;
	for (long long i = 0; i < 10 * ne + 6LL * m->nboundaryfaces; i++)
		if (m->elem2qnode[i] < 0 || m->elem2qnode[i] >= m->nbqnodes)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: elem2qnode index out of range");
	long long nbf = 0;
	for (long long F = 0; F < nf; F++) {
		const int eL = m->face2elem[4 * F], fL = m->face2elem[4 * F + 1], eR = m->face2elem[4 * F + 2],
				  fR = m->face2elem[4 * F + 3];
		if (eL < 0 || eL >= ne || fL < 0 || fL > 3 || eR >= ne || (eR >= 0 && (fR < 0 || fR > 3)))
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: face2elem entry out of range");
		if (eR < 0)
			nbf++;
	}
	if (nbf != m->nboundaryfaces)
		return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: nboundaryfaces does not match face2elem");
	return GDN_CUDA_OK;
}

static int validate_data(const gdn_cuda_data *d)
{
	if (!d || (d->kind != GDN_CUDA_DATA_PLANE && d->kind != GDN_CUDA_DATA_CAVITY &&
			   d->kind != GDN_CUDA_DATA_STATIONARY))
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: unknown analytic data kind");
	if (d->kind == GDN_CUDA_DATA_PLANE) {
		const double kk = d->khat[0] * d->khat[0] + d->khat[1] * d->khat[1] + d->khat[2] * d->khat[2];
		const double kp = d->khat[0] * d->pol[0] + d->khat[1] * d->pol[1] + d->khat[2] * d->pol[2];
		if (!(std::fabs(kk - 1.0) < 1e-12) || !(std::fabs(kp) < 1e-12) || !std::isfinite(d->kmag) ||
			!std::isfinite(d->amp) || !std::isfinite(d->phase))
			return gdn_set_error(GDN_CUDA_ERR_INVALID,
								 "attach: plane wave needs a unit direction and a polarisation orthogonal to it");
	}
	return GDN_CUDA_OK;
}

// neighbour / permutation / boundary tables from face2elem + fnode2enode
static int build_neighbours(const gdn_cuda_mesh *m, const gdn_cuda_tables *t, std::vector<int> &nb,
							std::vector<int> &perm, std::vector<double> &bxyz)
{
	const long long ne = m->nbelems, nf = m->nbfaces, nbf = m->nboundaryfaces;
	nb.assign(4 * ne, INT32_MIN);
	perm.assign(4 * ne, 0);
	bxyz.assign(nbf * 18, 0.0);
	std::vector<long long> bidx(nf, -1);
	for (long long b = 0; b < nbf; b++) {
		const int F = m->boundaryface[b];
		if (F < 0 || F >= nf || m->face2elem[4LL * F + 2] >= 0)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: boundaryface lists a non-boundary face");
		bidx[F] = b;
	}
	for (long long F = 0; F < nf; F++) {
		const int eL = m->face2elem[4 * F], fL = m->face2elem[4 * F + 1], eR = m->face2elem[4 * F + 2],
				  fR = m->face2elem[4 * F + 3];
		const int *fn = m->fnode2enode + 12 * F;
		for (int j = 0; j < 6; j++)
			if (fn[j] != t->face2node[fL][j])
				return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: fnode2enode (L side) disagrees with face2node");
		if (nb[4LL * eL + fL] != INT32_MIN)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: element face listed twice");
		if (eR < 0) {
			const long long b = bidx[F];
			if (b < 0)
				return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: boundary face missing from boundaryface");
			nb[4LL * eL + fL] = (int)(-(b + 1));
			for (int j = 0; j < 6; j++) {
				const long long q = m->elem2qnode[10LL * eL + fn[j]];
				for (int c = 0; c < 3; c++)
					bxyz[(b * 6 + j) * 3 + c] = m->node[3 * q + c];
			}
			continue;
		}
		if (nb[4LL * eR + fR] != INT32_MIN)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: element face listed twice");
		nb[4LL * eL + fL] = eR;
		nb[4LL * eR + fR] = eL;
		int pL = 0, pR = 0;
		for (int j = 0; j < 6; j++) {
			const int qr = fn[6 + j];
			if (qr < 0 || qr > 9)
				return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: fnode2enode (R side) out of range");
			pL |= qr << (4 * j);
		}
		for (int j = 0; j < 6; j++) {
			const int qself = t->face2node[fR][j];
			int jj = 0;
			while (jj < 6 && fn[6 + jj] != qself)
				jj++;
			if (jj == 6)
				return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: faces of neighbours do not match");
			pR |= fn[jj] << (4 * j);
		}
		perm[4LL * eL + fL] = pL;
		perm[4LL * eR + fR] = pR;
	}
	for (long long i = 0; i < 4 * ne; i++)
		if (nb[i] == INT32_MIN)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: an element face has no face record");
	return GDN_CUDA_OK;
}

template <typename S>
static S *as(void *p)
{
	return reinterpret_cast<S *>(p);
}

static const double RK_A[3] = {0., -5. / 9., -153. / 128.};
static const double RK_B[3] = {1. / 3., 15. / 16., 8. / 15.};
static const double RK_C[3] = {0., 1. / 3., 3. / 4.};

// RK3 stage-kernel autotuner: times both work decompositions on the handle's
// own buffers (contents are irrelevant to the timing; init / set_state
// rewrite them) and keeps the faster one.  Decisions are cached per
// (precision, floor(log2 ne)) for the life of the process.
static std::mutex g_tune_mu;
static std::map<std::pair<int, int>, int> g_tune;

template <typename T>
static int autotune_rk3(gdn_cuda_handle *h)
{
	int bucket = 0;
	while ((2LL << bucket) <= h->ne)
		bucket++;
	const std::pair<int, int> key(h->precision, bucket);
	{
		std::lock_guard<std::mutex> g(g_tune_mu);
		auto it = g_tune.find(key);
		if (it != g_tune.end()) {
			h->rk3_variant = it->second;
			return GDN_CUDA_OK;
		}
	}
	Rk3Params<T> p;
	p.w_in = as<T>(h->w[0]);
	p.w_out = as<T>(h->w[1]);
	p.k2 = as<T>(h->k2);
	p.geom = reinterpret_cast<const T *>(h->geomT);
	p.nb = h->nb;
	p.perm = h->perm;
	p.btrace = as<T>(h->btrace);
	p.einst = h->einst;
	p.dt_tab = h->dt_dev;
	p.ne = h->ne;
	p.dt = h->hdt[0];
	p.A = RK_A[1];
	p.B = RK_B[1];
	p.stage0 = 0;
	p.write_k2 = 1;
	p.sparse = h->rk3_sparse;
	p.fact = h->rk3_fact;
	p.num_sms = h->num_sms;
	p.idx32 = (h->ne + 31) / 32 * 1920 <= 0xffffffffLL;
	p.l2_ahead = 1;
	p.bc_metal = h->bc_metal;
	cudaEvent_t ev[2];
	GDN_CUDA_TRY(cudaEventCreate(&ev[0]));
	GDN_CUDA_TRY(cudaEventCreate(&ev[1]));
	float best = 0.f;
	int pick = 0;
	int rc = GDN_CUDA_OK;
	for (int v = 0; v < 2 && rc == GDN_CUDA_OK; v++) {
		float ms = 0.f;
		for (int rep = 0; rep < 4 && rc == GDN_CUDA_OK; rep++) { // launch 0 warms up
			if (rep == 1)
				cudaEventRecord(ev[0], h->stream);
			rc = launch_rk3_stage<T>(p, v, h->stream);
			h->launches++;
		}
		if (rc != GDN_CUDA_OK)
			break;
		cudaEventRecord(ev[1], h->stream);
		cudaError_t e = cudaEventSynchronize(ev[1]);
		if (e == cudaSuccess)
			e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
		if (e != cudaSuccess)
			rc = gdn_cuda_fail(e, "autotune_rk3", __FILE__, __LINE__);
		if (v == 0 || ms < best) {
			best = ms;
			pick = v;
		}
	}
	cudaEventDestroy(ev[0]);
	cudaEventDestroy(ev[1]);
	if (rc != GDN_CUDA_OK)
		return rc;
	h->rk3_variant = pick;
	std::lock_guard<std::mutex> g(g_tune_mu);
	g_tune[key] = pick;
	return GDN_CUDA_OK;
}

static int kin_prepare_grids(gdn_cuda_handle *h);
static int kin_prepare_parts(gdn_cuda_handle *h, const gdn_cuda_mesh *m);
static int autotune_kin(gdn_cuda_handle *h);

static int attach_impl(gdn_cuda_handle *h, const gdn_cuda_mesh *m, const gdn_cuda_tables *t,
					   const gdn_cuda_model *mo)
{
	const long long ne = h->ne, nf = h->nf, nbf = h->nbf;
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	GDN_CUDA_TRY(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
	// The kinetic step is a chain of small dependent sweep launches whose
	// time is latency: its stream gets the highest priority, so that its CTAs
	// are dispatched ahead of pending CTAs of throughput work (an RK3 batch)
	// sharing the GPU.
	int least = 0, greatest = 0;
	GDN_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
	GDN_CUDA_TRY(cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking,
											  h->scheme == GDN_CUDA_SCHEME_KINETIC ? greatest : least));
	if (!rk3_tables_standard_faces(t))
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "attach: face2node differs from the P2 convention");
	h->rk3_sparse = rk3_tables_sparse(t) ? 1 : 0;
	h->rk3_fact = h->rk3_sparse && rk3_tables_factor(t) ? 1 : 0;
	GDN_TRY(upload_tables(t));
	std::vector<int> nb, perm;
	std::vector<double> bx;
	GDN_TRY(build_neighbours(m, t, nb, perm, bx));

	GDN_TRY(dalloc(h, &h->e2q, 10 * ne));
	GDN_TRY(dalloc(h, &h->node, 3 * h->nq));
	GDN_TRY(dalloc(h, &h->geom64, 10 * ne));
	GDN_TRY(dalloc(h, &h->nb, 4 * ne));
	GDN_TRY(dalloc(h, &h->perm, 4 * ne));
	GDN_TRY(dalloc(h, &h->face2elem, 4 * nf));
	GDN_TRY(dalloc(h, &h->bxyz, 18 * (nbf > 0 ? nbf : 1)));
	GDN_TRY(dalloc(h, &h->flag, 4));
	h->nblk_err = 1184; // 8 x 148 SMs
	GDN_TRY(dalloc(h, &h->partial, 6 * h->nblk_err));
	GDN_TRY(dalloc(h, &h->result, 8));
	GDN_TRY(dalloc(h, &h->t_dev, h->ninst));
	GDN_TRY(dalloc(h, &h->dt_dev, h->ninst));
	GDN_TRY(dalloc(h, &h->data_dev, h->ninst));
	GDN_CUDA_TRY(cudaMallocHost(&h->host_result, 8 * sizeof(double)));
	cudaStream_t s = h->stream;
	GDN_CUDA_TRY(cudaMemcpyAsync(h->dt_dev, h->hdt.data(), h->ninst * sizeof(double), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(
		cudaMemcpyAsync(h->data_dev, h->hdata.data(), h->ninst * sizeof(Data), cudaMemcpyHostToDevice, s));
	if (h->ninst > 1) {
		std::vector<int> ei(ne), bi(nbf > 0 ? nbf : 1);
		for (int i = 0; i < h->ninst; i++) {
			for (long long e = h->e_off[i]; e < h->e_off[i + 1]; e++)
				ei[e] = i;
			for (long long b = h->bf_off[i]; b < h->bf_off[i + 1]; b++)
				bi[b] = i;
		}
		GDN_TRY(dalloc(h, &h->einst, ne));
		GDN_TRY(dalloc(h, &h->bfinst, bi.size()));
		GDN_CUDA_TRY(cudaMemcpyAsync(h->einst, ei.data(), ne * sizeof(int), cudaMemcpyHostToDevice, s));
		GDN_CUDA_TRY(cudaMemcpyAsync(h->bfinst, bi.data(), bi.size() * sizeof(int), cudaMemcpyHostToDevice, s));
		GDN_CUDA_TRY(cudaStreamSynchronize(s)); // the host vectors go out of scope
	}
	GDN_CUDA_TRY(cudaMemcpyAsync(h->e2q, m->elem2qnode, 10 * ne * sizeof(int), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(h->node, m->node, 3 * h->nq * sizeof(double), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(h->nb, nb.data(), 4 * ne * sizeof(int), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(h->perm, perm.data(), 4 * ne * sizeof(int), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(h->face2elem, m->face2elem, 4 * nf * sizeof(int), cudaMemcpyHostToDevice, s));
	if (nbf > 0)
		GDN_CUDA_TRY(cudaMemcpyAsync(h->bxyz, bx.data(), 18 * nbf * sizeof(double), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemsetAsync(h->flag, 0, 4 * sizeof(int), s));
	GDN_TRY(launch_geometry(h->e2q, h->node, ne, h->geom64, h->flag, s));
	h->launches++;
	int bad = 0;
	GDN_CUDA_TRY(cudaMemcpyAsync(&bad, h->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	if (bad)
		return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: an element has a non-positive Jacobian determinant");

	const bool fp64 = h->precision == GDN_CUDA_FP64;
	if (h->scheme == GDN_CUDA_SCHEME_RK3) {
		// state, k2 and geometry in tiles of 32 elements (the last one padded)
		const long long nt = 32 * ((ne + 31) / 32);
		h->neq = 10 * ne + 6 * nbf;
		if (fp64) {
			double *gt;
			GDN_TRY(dalloc(h, &gt, 10 * nt));
			GDN_TRY(launch_geom_to_tiles<double>(h->geom64, gt, ne, s));
			h->geomT = gt;
		} else {
			float *gt;
			GDN_TRY(dalloc(h, &gt, 10 * nt));
			GDN_TRY(launch_geom_to_tiles<float>(h->geom64, gt, ne, s));
			h->geomT = gt;
		}
		h->launches++;
		GDN_TRY(prepare_rk3<double>());
		GDN_TRY(prepare_rk3<float>());
		if (fp64)
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->btrace), 36 * (nbf > 0 ? nbf : 1)));
		else
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->btrace), 36 * (nbf > 0 ? nbf : 1)));
		for (int b = 0; b < 2; b++) {
			if (fp64)
				GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->w[b]), 60 * nt));
			else
				GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->w[b]), 60 * nt));
		}
		if (fp64)
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->k2), 60 * nt));
		else
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->k2), 60 * nt));
		GDN_CUDA_TRY(cudaMemsetAsync(h->k2, 0, 60 * nt * h->ssize, s));
		GDN_TRY(dalloc(h, &h->staging, 6 * h->neq));
		if (h->rk3_autotune) {
			GDN_CUDA_TRY(cudaMemsetAsync(h->w[0], 0, 60 * nt * h->ssize, s));
			GDN_CUDA_TRY(cudaMemsetAsync(h->btrace, 0, 36 * (nbf > 0 ? nbf : 1) * h->ssize, s));
			if (fp64)
				GDN_TRY(autotune_rk3<double>(h));
			else
				GDN_TRY(autotune_rk3<float>(h));
		}
	} else {
		const int nv = h->nv;
		h->neq = 10 * ne + 6 * nbf;
		const long long nu = ne * nv;
		unsigned char *mask;
		GDN_TRY(dalloc(h, &h->sown64, 4 * nu));
		GDN_TRY(dalloc(h, &mask, nu));
		// upwind masks first: the schedule (and with it the sweep order every
		// other kinetic array is stored in) is built on the device from them
		GDN_TRY(launch_kin_setup<double>(h->face2elem, nf, h->geom64, h->nb, ne, h->km, h->sown64, mask, s));
		h->launches += 2;
		GDN_TRY(dalloc(h, &h->items, nu));
		GDN_TRY(dalloc(h, &h->pos, nu));
		GDN_TRY(dalloc(h, &h->rnb, nu));
		GDN_TRY(dalloc(h, &h->rpm, nu));
		GDN_TRY(dalloc(h, &h->bt, 36LL * nv * (nbf > 0 ? nbf : 1)));
		GDN_TRY(kin_device_schedule(mask, h->nb, h->sown64, ne, nv, h->items, h->pos, h->level_off, h->spin_limit, s));
		h->launches += 4;
		// state f: FP64 for FP64 and FP32_REFINE, FP32, or BF16
		if (h->precision == GDN_CUDA_FP64 || h->precision == GDN_CUDA_FP32_REFINE)
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->f), 60 * nu));
		else if (h->precision == GDN_CUDA_FP32)
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->f), 60 * nu));
		else
			GDN_TRY(dalloc(h, reinterpret_cast<__nv_bfloat16 **>(&h->f), 60 * nu));
		if (h->precision == GDN_CUDA_FP32_REFINE) {
			GDN_TRY(dalloc(h, &h->yacc, 60 * nu));
			GDN_TRY(dalloc(h, &h->rhs, 60 * nu));
			GDN_TRY(dalloc(h, &h->ru64, nu));
			GDN_TRY(dalloc(h, &h->rs64, nu));
		}
		GDN_TRY(kin_upload_block_tables(t));
		if (fp64) {
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->G), 100 * nu));
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->rs), 4 * nu));
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->rcoef), nu));
			GDN_TRY(dalloc(h, reinterpret_cast<double **>(&h->y), 60 * nu));
			GDN_TRY(launch_kin_blocks<double>(h->geom64, h->sown64, h->items, h->pos, h->nb, h->perm, ne, h->km,
											  h->theta, h->einst, h->dt_dev, as<double>(h->G), as<double>(h->rcoef), h->rnb,
											  h->rpm, as<double>(h->rs), h->ru64, h->rs64, h->flag, s));
		} else {
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->G), 100 * nu));
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->rs), 4 * nu));
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->rcoef), nu));
			GDN_TRY(dalloc(h, reinterpret_cast<float **>(&h->y), 60 * nu));
			GDN_TRY(launch_kin_blocks<float>(h->geom64, h->sown64, h->items, h->pos, h->nb, h->perm, ne, h->km,
											 h->theta, h->einst, h->dt_dev, as<float>(h->G), as<float>(h->rcoef), h->rnb, h->rpm,
											 as<float>(h->rs), h->ru64, h->rs64, h->flag, s));
		}
		h->launches += 2;
		GDN_CUDA_TRY(cudaMemcpyAsync(&bad, h->flag, sizeof(int), cudaMemcpyDeviceToHost, s));
		GDN_CUDA_TRY(cudaStreamSynchronize(s));
		if (bad)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "attach: a transport diagonal block is singular");
		GDN_TRY(dalloc(h, &h->staging, (long long)6 * nv * h->neq));
		// the cooperative sweep: level table, barrier, error flag, grids
		const int nl = (int)h->level_off.size() - 1;
		GDN_TRY(dalloc(h, &h->level_off_dev, nl + 1));
		GDN_CUDA_TRY(cudaMemcpyAsync(h->level_off_dev, h->level_off.data(), (nl + 1) * sizeof(int),
									 cudaMemcpyHostToDevice, s));
		GDN_TRY(dalloc(h, &h->bar, 2));
		GDN_TRY(dalloc(h, &h->err, 1));
		GDN_CUDA_TRY(cudaMemsetAsync(h->bar, 0, 2 * sizeof(unsigned), s));
		GDN_CUDA_TRY(cudaMemsetAsync(h->err, 0, sizeof(int), s));
		// the flag-driven sweep: level-aligned chunks in sweep order
		std::vector<int2> chunks;
		for (int l = 0; l < nl; l++) {
			const int nch = (h->level_off[l + 1] - h->level_off[l] + 31) / 32;
			h->max_chunks = nch > h->max_chunks ? nch : h->max_chunks;
			for (int k0 = h->level_off[l]; k0 < h->level_off[l + 1]; k0 += 32)
				chunks.push_back(make_int2(k0, k0 + 32 < h->level_off[l + 1] ? k0 + 32 : h->level_off[l + 1]));
		}
		h->nchunks = (int)chunks.size();
		GDN_TRY(dalloc(h, &h->kchunks, chunks.size()));
		GDN_CUDA_TRY(cudaMemcpyAsync(h->kchunks, chunks.data(), chunks.size() * sizeof(int2), cudaMemcpyHostToDevice,
									 s));
		GDN_TRY(dalloc(h, &h->kready, nu));
		GDN_TRY(dalloc(h, &h->kqueue, 1));
		GDN_TRY(kin_prepare_grids(h));
		GDN_TRY(kin_prepare_parts(h, m));
		GDN_CUDA_TRY(cudaStreamSynchronize(s));
		if (h->kin_autotune)
			GDN_TRY(autotune_kin(h));
	}
	return GDN_CUDA_OK;
}

static Data to_data(const gdn_cuda_data *d)
{
	Data o;
	o.kind = d->kind;
	for (int c = 0; c < 3; c++) {
		o.khat[c] = d->khat[c];
		o.pol[c] = d->pol[c];
	}
	o.kmag = d->kmag;
	o.amp = d->amp;
	o.phase = d->phase;
	return o;
}

static int validate_model(const gdn_cuda_model *model, const gdn_cuda_config &cfg)
{
	if (!model)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: model missing");
	if (model->nb_w != 6)
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "attach: only Maxwell (nb_w = 6) runs on the device");
	if (model->scheme != GDN_CUDA_SCHEME_RK3 && model->scheme != GDN_CUDA_SCHEME_KINETIC)
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "attach: unknown scheme");
	if (model->scheme == GDN_CUDA_SCHEME_RK3 && cfg.precision > GDN_CUDA_FP32)
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "attach: RK3 supports FP64 and FP32");
	if (model->boundary_flux != GDN_CUDA_BC_UPWIND && model->boundary_flux != GDN_CUDA_BC_METAL)
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "attach: unknown boundary flux");
	if (model->scheme == GDN_CUDA_SCHEME_KINETIC && model->boundary_flux != GDN_CUDA_BC_UPWIND)
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED,
							 "attach: the kinetic scheme imposes f_eq of the data on boundaries (upwind only)");
	if (model->scheme == GDN_CUDA_SCHEME_KINETIC) {
		if (model->nb_v != 4 && model->nb_v != 6)
			return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "attach: kinetic sets d3q4 (4) or d3q6 (6) only");
		if (!model->vi || !(model->lambda > 0.0) || !(model->theta > 0.0) || !(model->theta <= 1.0))
			return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: kinetic model needs vi, lambda > 0, 0 < theta <= 1");
		if (cfg.precision == GDN_CUDA_FP32_REFINE && (cfg.refine_passes < 0 || cfg.refine_passes > 4))
			return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: refine_passes must be in [0, 4]");
	}
	return GDN_CUDA_OK;
}

// instances of one batch share the scheme and, for the kinetic scheme, the
// whole velocity model (one relaxation kernel serves them all)
static bool same_model(const gdn_cuda_model *a, const gdn_cuda_model *b)
{
	if (a->scheme != b->scheme || a->boundary_flux != b->boundary_flux)
		return false;
	if (a->scheme == GDN_CUDA_SCHEME_RK3)
		return true;
	if (a->nb_v != b->nb_v || a->lambda != b->lambda || a->omega != b->omega || a->theta != b->theta)
		return false;
	for (int i = 0; i < 3 * a->nb_v; i++)
		if (a->vi[i] != b->vi[i])
			return false;
	return true;
}

// host arrays of the concatenated mesh of a batch
struct MeshCat {
	std::vector<int> face2elem, fnode2enode, boundaryface, elem2qnode;
	std::vector<double> node;
	gdn_cuda_mesh m{};
};

static int concat_meshes(const gdn_cuda_instance *inst, int n, gdn_cuda_handle *h, MeshCat &mc)
{
	long long ne = 0, nf = 0, nbf = 0, nq = 0;
	for (int i = 0; i < n; i++) {
		ne += inst[i].mesh->nbelems;
		nf += inst[i].mesh->nbfaces;
		nbf += inst[i].mesh->nboundaryfaces;
		nq += inst[i].mesh->nbqnodes;
	}
	if (ne > (1LL << 28) || nf > (1LL << 29) || nq > (1LL << 29))
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: batch too large for 32-bit element / node indices");
	mc.face2elem.resize(4 * nf);
	mc.fnode2enode.resize(12 * nf);
	mc.boundaryface.resize(nbf);
	mc.elem2qnode.resize(10 * ne + 6 * nbf);
	mc.node.resize(3 * nq);
	long long e0 = 0, f0 = 0, b0 = 0, q0 = 0;
	h->e_off.assign(1, 0);
	h->q_off.assign(1, 0);
	h->bf_off.assign(1, 0);
	for (int i = 0; i < n; i++) {
		const gdn_cuda_mesh *m = inst[i].mesh;
		for (long long F = 0; F < m->nbfaces; F++) {
			const int *src = m->face2elem + 4 * F;
			int *dst = mc.face2elem.data() + 4 * (f0 + F);
			dst[0] = (int)(src[0] + e0);
			dst[1] = src[1];
			dst[2] = src[2] >= 0 ? (int)(src[2] + e0) : src[2];
			dst[3] = src[3];
		}
		std::memcpy(mc.fnode2enode.data() + 12 * f0, m->fnode2enode, 12 * (size_t)m->nbfaces * sizeof(int));
		for (long long b = 0; b < m->nboundaryfaces; b++)
			mc.boundaryface[b0 + b] = (int)(m->boundaryface[b] + f0);
		for (long long v = 0; v < 10LL * m->nbelems; v++)
			mc.elem2qnode[10 * e0 + v] = (int)(m->elem2qnode[v] + q0);
		for (long long v = 0; v < 6LL * m->nboundaryfaces; v++)
			mc.elem2qnode[10 * ne + 6 * b0 + v] = (int)(m->elem2qnode[10LL * m->nbelems + v] + q0);
		std::memcpy(mc.node.data() + 3 * q0, m->node, 3 * (size_t)m->nbqnodes * sizeof(double));
		e0 += m->nbelems;
		f0 += m->nbfaces;
		b0 += m->nboundaryfaces;
		q0 += m->nbqnodes;
		h->q_off.push_back(q0);
		h->e_off.push_back(e0);
		h->bf_off.push_back(b0);
	}
	mc.m.nbelems = (int)ne;
	mc.m.nbfaces = (int)nf;
	mc.m.nboundaryfaces = (int)nbf;
	mc.m.nbqnodes = (int)nq;
	mc.m.face2elem = mc.face2elem.data();
	mc.m.fnode2enode = mc.fnode2enode.data();
	mc.m.boundaryface = mc.boundaryface.data();
	mc.m.elem2qnode = mc.elem2qnode.data();
	mc.m.node = mc.node.data();
	return GDN_CUDA_OK;
}

static int attach_batch(const gdn_cuda_instance *inst, int n, const gdn_cuda_tables *tables,
						const gdn_cuda_config *config, gdn_cuda_handle **out)
{
	if (!out)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: out is NULL");
	*out = nullptr;
	if (!inst || n <= 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: no instances");
	if (!tables)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: tables missing");
	gdn_cuda_config cfg = {GDN_CUDA_FP64, 1, 0, 1, 0, 0};
	if (config)
		cfg = *config;
	if (cfg.precision < GDN_CUDA_FP64 || cfg.precision > GDN_CUDA_BF16_STORE)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: unknown precision mode");
	if (cfg.rk3_variant < 0 || cfg.rk3_variant > 2)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: rk3_variant must be 0 (auto), 1 or 2");
	if (cfg.kin_sweep < 0 || cfg.kin_sweep > 4)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: kin_sweep must be 0 (auto), 1, 2, 3 or 4");
	for (int i = 0; i < n; i++) {
		GDN_TRY(validate_mesh(inst[i].mesh));
		GDN_TRY(validate_data(inst[i].data));
		GDN_TRY(validate_model(inst[i].model, cfg));
		if (!(inst[i].dt > 0.0) || !std::isfinite(inst[i].dt))
			return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: dt must be positive");
		if (!same_model(inst[0].model, inst[i].model))
			return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED,
								 "attach: the instances of a batch need one scheme and one kinetic model");
	}
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
		cudaGetLastError();
		return gdn_set_error(GDN_CUDA_ERR_CUDA, "attach: no CUDA device");
	}
	if (cfg.device < 0 || cfg.device >= ndev)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "attach: bad device ordinal");

	const gdn_cuda_model *model = inst[0].model;
	gdn_cuda_handle *h = new gdn_cuda_handle();
	h->device = cfg.device;
	h->scheme = model->scheme;
	h->precision = cfg.precision;
	h->refine_passes = cfg.refine_passes;
	h->use_graph = cfg.use_graph;
	// RK3 stage kernel compiled for fewer (1) or more (2) resident CTAs per
	// SM; 0 = timed at attach
	h->rk3_variant = cfg.rk3_variant > 0 ? cfg.rk3_variant - 1 : 0;
	h->rk3_autotune = cfg.rk3_variant == 0;
	h->kin_mode = cfg.kin_sweep == 0 ? 1 : cfg.kin_sweep;
	h->kin_autotune = cfg.kin_sweep == 0;
	h->ninst = n;
	for (int i = 0; i < n; i++) {
		h->hdata.push_back(to_data(inst[i].data));
		h->hdt.push_back(inst[i].dt);
	}
	h->ht.assign(n, 0.0);
	h->ht_bdof.assign(n, 0.0);
	h->theta = model->theta > 0 ? model->theta : 0.5;
	h->omega = model->omega;
	h->lambda = model->lambda;
	h->bc_metal = model->boundary_flux == GDN_CUDA_BC_METAL;
	h->ssize = cfg.precision == GDN_CUDA_FP64 ? 8 : 4;
	if (h->scheme == GDN_CUDA_SCHEME_KINETIC) {
		h->nv = model->nb_v;
		h->km.nv = h->nv;
		for (int i = 0; i < 3 * h->nv; i++)
			h->km.vi[i] = model->vi[i];
		const double l2 = model->lambda * model->lambda;
		h->km.feq_c = h->nv == 4 ? 1.0 / (4.0 * l2) : 1.0 / (2.0 * l2);
	}
	MeshCat mc;
	const gdn_cuda_mesh *mesh = inst[0].mesh;
	int rc = GDN_CUDA_OK;
	if (n > 1) {
		rc = concat_meshes(inst, n, h, mc);
		mesh = &mc.m;
	} else {
		h->e_off = {0, mesh->nbelems};
		h->q_off = {0, mesh->nbqnodes};
		h->bf_off = {0, mesh->nboundaryfaces};
	}
	if (rc == GDN_CUDA_OK) {
		const long long m = h->scheme == GDN_CUDA_SCHEME_RK3 ? 6 : 6LL * h->nv;
		h->w_off.assign(1, 0);
		for (int i = 0; i < n; i++) {
			const long long neq = 10 * (h->e_off[i + 1] - h->e_off[i]) + 6 * (h->bf_off[i + 1] - h->bf_off[i]);
			h->neq_i.push_back(neq);
			h->w_off.push_back(h->w_off.back() + m * neq);
		}
		h->ne = mesh->nbelems;
		h->nf = mesh->nbfaces;
		h->nbf = mesh->nboundaryfaces;
		h->nq = mesh->nbqnodes;
		rc = attach_impl(h, mesh, tables, model);
	}
	if (rc != GDN_CUDA_OK) {
		std::string msg = g_last_error;
		free_handle(h);
		g_last_error = msg;
		return rc;
	}
	*out = h;
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_attach(const gdn_cuda_mesh *mesh, const gdn_cuda_tables *tables,
							   const gdn_cuda_model *model, const gdn_cuda_data *data,
							   const gdn_cuda_config *config, double dt, gdn_cuda_handle **out)
{
	gdn_cuda_instance one;
	one.mesh = mesh;
	one.model = model;
	one.data = data;
	one.dt = dt;
	return attach_batch(&one, 1, tables, config, out);
}

extern "C" int gdn_cuda_attach_batch(const gdn_cuda_instance *inst, int ninst, const gdn_cuda_tables *tables,
									 const gdn_cuda_config *config, gdn_cuda_handle **out)
{
	return attach_batch(inst, ninst, tables, config, out);
}

extern "C" int gdn_cuda_detach(gdn_cuda_handle *h)
{
	if (!h)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "detach: NULL handle");
	free_handle(h);
	return GDN_CUDA_OK;
}

// ------------------------------------------------------------ stepping --

// ---- enqueue one time step (no host bookkeeping; capturable) ----
template <typename T>
static int rk3_enqueue(gdn_cuda_handle *h, int &cur, long long &nlaunch)
{
	const Batch bt = h->batch();
	for (int i = 0; i < 3; i++) {
		Rk3Params<T> p;
		p.w_in = as<T>(h->w[cur]);
		p.w_out = as<T>(h->w[1 - cur]);
		p.k2 = as<T>(h->k2);
		p.geom = reinterpret_cast<const T *>(h->geomT);
		p.nb = h->nb;
		p.perm = h->perm;
		p.btrace = as<T>(h->btrace);
		p.einst = h->einst;
		p.dt_tab = h->dt_dev;
		p.ne = h->ne;
		p.dt = h->hdt[0];
		p.A = RK_A[i];
		p.B = RK_B[i];
		p.stage0 = i == 0;
		p.write_k2 = i < 2;
		p.sparse = h->rk3_sparse;
		p.fact = h->rk3_fact;
		p.num_sms = h->num_sms;
		p.idx32 = (h->ne + 31) / 32 * 1920 <= 0xffffffffLL;
		p.l2_ahead = 1;
		p.bc_metal = h->bc_metal;
		if (h->nbf > 0) {
			GDN_TRY(launch_boundary_trace<T>(h->bxyz, h->nbf, bt, RK_C[i], as<T>(h->btrace), h->stream));
			nlaunch++;
		}
		GDN_TRY(launch_rk3_stage<T>(p, h->rk3_variant, h->stream));
		nlaunch++;
		cur = 1 - cur;
	}
	GDN_TRY(launch_advance_time(bt, h->stream));
	nlaunch++;
	return GDN_CUDA_OK;
}

// all sweep levels of one transport solve M1 y = f
template <typename F, typename Y, typename T>
static int kin_sweeps(gdn_cuda_handle *h, const void *f, int acc, int bdata, long long &nlaunch)
{
	KinSweepParams p;
	p.f = f;
	p.y = h->y;
	p.yacc = h->yacc;
	p.G = h->G;
	p.rs = h->rs;
	p.rcoef = h->rcoef;
	p.rnb = h->rnb;
	p.rpm = h->rpm;
	p.items = h->items;
	p.bt = h->bt;
	p.nv = h->nv;
	const int nl = (int)h->level_off.size() - 1;
	if (h->kin_mode == 2) {
		int grid = h->kin_grid[acc] < h->max_chunks ? h->kin_grid[acc] : h->max_chunks;
		grid = grid > 0 ? grid : 1;
		p.item_begin = 0;
		p.item_end = h->level_off[nl];
		GDN_TRY((launch_kin_levels<F, Y, T>(p, h->level_off_dev, nl, grid, h->bar, h->err, h->spin_limit, acc, bdata,
											h->rk3_sparse, h->stream)));
		nlaunch++;
		return GDN_CUDA_OK;
	}
	if (h->kin_mode == 4) {
		p.item_begin = 0;
		p.item_end = h->level_off[nl];
		GDN_TRY((launch_kin_parts<F, Y, T>(p, h->plist, h->pchunks, h->part_chunk_off, h->nparts, h->kready,
										   h->ne * h->nv, h->err, h->spin_limit, acc, bdata, h->rk3_sparse,
										   h->stream)));
		nlaunch++;
		return GDN_CUDA_OK;
	}
	if (h->kin_mode == 3) {
		p.item_begin = 0;
		p.item_end = h->level_off[nl];
		GDN_TRY((launch_kin_flags<F, Y, T>(p, h->kchunks, h->nchunks, h->kin_fgrid[acc] > 0 ? h->kin_fgrid[acc] : 1,
										   h->kqueue, h->kready, h->ne * h->nv, h->err, h->spin_limit, acc, bdata,
										   h->rk3_sparse, h->stream)));
		nlaunch++;
		return GDN_CUDA_OK;
	}
	for (int l = 0; l < nl; l++) {
		p.item_begin = h->level_off[l];
		p.item_end = h->level_off[l + 1];
		GDN_TRY((launch_kin_sweep<F, Y, T>(p, acc, bdata, h->rk3_sparse, h->stream)));
		nlaunch++;
	}
	return GDN_CUDA_OK;
}

template <typename F, typename Y, typename T>
static int kin_relax(gdn_cuda_handle *h, const void *y, long long &nlaunch)
{
	KinRelaxParams r;
	r.f = h->f;
	r.y = y;
	r.pos = h->pos;
	r.ne = h->ne;
	r.nv = h->nv;
	for (int i = 0; i < 3 * NV_MAX; i++)
		r.vi[i] = h->km.vi[i];
	r.feq_c = h->km.feq_c;
	r.omega = h->omega;
	r.a_y = 1.0 / h->theta;
	r.a_f = -(1.0 - h->theta) / h->theta;
	GDN_TRY((launch_kin_relax<F, Y, T>(r, h->stream)));
	nlaunch++;
	return GDN_CUDA_OK;
}

// one CFL-less step: boundary f_eq at t + dt/2, the transport solve of every
// velocity (level sweeps), the relaxation, t += dt
static int kin_enqueue(gdn_cuda_handle *h, long long &nlaunch)
{
	if (h->nbf > 0) {
		GDN_TRY(launch_kin_boundary_trace(h->bxyz, h->nbf, h->batch(), h->nv, h->km.vi, h->km.feq_c, h->bt,
										  h->stream));
		nlaunch++;
	}
	switch (h->precision) {
	case GDN_CUDA_FP64:
		GDN_TRY((kin_sweeps<double, double, double>(h, h->f, 0, 1, nlaunch)));
		GDN_TRY((kin_relax<double, double, double>(h, h->y, nlaunch)));
		break;
	case GDN_CUDA_FP32:
		GDN_TRY((kin_sweeps<float, float, float>(h, h->f, 0, 1, nlaunch)));
		GDN_TRY((kin_relax<float, float, float>(h, h->y, nlaunch)));
		break;
	case GDN_CUDA_BF16_STORE:
		GDN_TRY((kin_sweeps<__nv_bfloat16, float, float>(h, h->f, 0, 1, nlaunch)));
		GDN_TRY((kin_relax<__nv_bfloat16, float, float>(h, h->y, nlaunch)));
		break;
	default: { // GDN_CUDA_FP32_REFINE
		GDN_TRY((kin_sweeps<double, float, float>(h, h->f, 1, 1, nlaunch)));
		KinResidualParams q;
		q.f = as<double>(h->f);
		q.yacc = h->yacc;
		q.r = h->rhs;
		q.rnb = h->rnb;
		q.rpm = h->rpm;
		q.items = h->items;
		q.ru64 = h->ru64;
		q.rs64 = h->rs64;
		q.bt = h->bt;
		q.nv = h->nv;
		q.nitems = h->ne * h->nv;
		for (int pass = 0; pass < h->refine_passes; pass++) {
			GDN_TRY(launch_kin_residual(q, h->rk3_sparse, h->stream));
			nlaunch++;
			GDN_TRY((kin_sweeps<float, float, float>(h, h->rhs, 2, 0, nlaunch)));
		}
		GDN_TRY((kin_relax<double, double, double>(h, h->yacc, nlaunch)));
		break;
	}
	}
	GDN_TRY(launch_advance_time(h->batch(), h->stream));
	nlaunch++;
	return GDN_CUDA_OK;
}

// CTAs of the cooperative and the flag-driven sweeps for the variants this
// handle's precision runs
static int kin_prepare_flag_grids(gdn_cuda_handle *h)
{
	const int sp = h->rk3_sparse;
	switch (h->precision) {
	case GDN_CUDA_FP64:
		return kin_flags_grid<double, double, double>(h->device, 0, sp, &h->kin_fgrid[0]);
	case GDN_CUDA_FP32:
		return kin_flags_grid<float, float, float>(h->device, 0, sp, &h->kin_fgrid[0]);
	case GDN_CUDA_BF16_STORE:
		return kin_flags_grid<__nv_bfloat16, float, float>(h->device, 0, sp, &h->kin_fgrid[0]);
	default:
		GDN_TRY((kin_flags_grid<double, float, float>(h->device, 1, sp, &h->kin_fgrid[1])));
		return kin_flags_grid<float, float, float>(h->device, 2, sp, &h->kin_fgrid[2]);
	}
}

static int kin_prepare_grids(gdn_cuda_handle *h)
{
	const int sp = h->rk3_sparse;
	GDN_TRY(kin_prepare_flag_grids(h));
	switch (h->precision) {
	case GDN_CUDA_FP64:
		GDN_TRY((kin_parts_grid<double, double, double>(h->device, 0, sp, &h->kin_pgrid[0])));
		break;
	case GDN_CUDA_FP32:
		GDN_TRY((kin_parts_grid<float, float, float>(h->device, 0, sp, &h->kin_pgrid[0])));
		break;
	case GDN_CUDA_BF16_STORE:
		GDN_TRY((kin_parts_grid<__nv_bfloat16, float, float>(h->device, 0, sp, &h->kin_pgrid[0])));
		break;
	default:
		GDN_TRY((kin_parts_grid<double, float, float>(h->device, 1, sp, &h->kin_pgrid[1])));
		GDN_TRY((kin_parts_grid<float, float, float>(h->device, 2, sp, &h->kin_pgrid[2])));
	}
	switch (h->precision) {
	case GDN_CUDA_FP64:
		return kin_levels_grid<double, double, double>(h->device, 0, sp, &h->kin_grid[0]);
	case GDN_CUDA_FP32:
		return kin_levels_grid<float, float, float>(h->device, 0, sp, &h->kin_grid[0]);
	case GDN_CUDA_BF16_STORE:
		return kin_levels_grid<__nv_bfloat16, float, float>(h->device, 0, sp, &h->kin_grid[0]);
	default:
		GDN_TRY((kin_levels_grid<double, float, float>(h->device, 1, sp, &h->kin_grid[1])));
		return kin_levels_grid<float, float, float>(h->device, 2, sp, &h->kin_grid[2]);
	}
}

// The spatial parts of the parts sweep: as many parts as CTAs of every
// launched variant fit at once (at least 32 elements each), the item list by
// part (device), its level-aligned chunks (at most 32 items) and each part's
// chunk range.
static int kin_prepare_parts(gdn_cuda_handle *h, const gdn_cuda_mesh *m)
{
	int cap = 0;
	for (int a = 0; a < 3; a++)
		if (h->kin_pgrid[a] > 0)
			cap = cap == 0 || h->kin_pgrid[a] < cap ? h->kin_pgrid[a] : cap;
	const long long byelem = h->ne / 32 > 0 ? h->ne / 32 : 1;
	h->nparts = (int)(cap < byelem ? cap : byelem);
	if (h->nparts < 1)
		h->nparts = 1;
	double lo[3] = {m->node[0], m->node[1], m->node[2]}, hi[3] = {m->node[0], m->node[1], m->node[2]};
	for (long long q = 0; q < h->nq; q++)
		for (int a = 0; a < 3; a++) {
			lo[a] = std::fmin(lo[a], m->node[3 * q + a]);
			hi[a] = std::fmax(hi[a], m->node[3 * q + a]);
		}
	const long long nitems = h->ne * h->nv;
	GDN_TRY(dalloc(h, &h->plist, nitems));
	std::vector<int> plist, pkey;
	GDN_TRY(kin_build_parts(h->e2q, h->node, h->ne, lo, hi, h->items, nitems, h->nv, h->nparts, h->rnb, h->rpm,
							h->plist, plist, pkey, h->stream));
	h->launches += 5;
	std::vector<int2> chunks;
	std::vector<int> off(h->nparts + 1, 0);
	long long i = 0;
	for (int b = 0; b < h->nparts; b++) {
		off[b] = (int)chunks.size();
		size_t l = 0; // level of the current item (plist is in sweep order within a part)
		int start = -1, cnt = 0;
		size_t lstart = 0;
		for (; i < nitems && pkey[i] == b; i++) {
			const int k = plist[i];
			while (l + 1 < h->level_off.size() && k >= h->level_off[l + 1])
				l++;
			if (start < 0 || l != lstart || cnt == 32) {
				if (start >= 0)
					chunks.push_back(make_int2(start, cnt));
				start = (int)i;
				cnt = 0;
				lstart = l;
			}
			cnt++;
		}
		if (start >= 0)
			chunks.push_back(make_int2(start, cnt));
	}
	off[h->nparts] = (int)chunks.size();
	GDN_TRY(dalloc(h, &h->pchunks, chunks.size()));
	GDN_TRY(dalloc(h, &h->part_chunk_off, off.size()));
	GDN_CUDA_TRY(cudaMemcpyAsync(h->pchunks, chunks.data(), chunks.size() * sizeof(int2), cudaMemcpyHostToDevice,
								 h->stream));
	GDN_CUDA_TRY(cudaMemcpyAsync(h->part_chunk_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice,
								 h->stream));
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	return GDN_CUDA_OK;
}

// the first transport solve of a step, as the step runs it
static int kin_first_sweep(gdn_cuda_handle *h, long long &nl)
{
	switch (h->precision) {
	case GDN_CUDA_FP64:
		return kin_sweeps<double, double, double>(h, h->f, 0, 1, nl);
	case GDN_CUDA_FP32:
		return kin_sweeps<float, float, float>(h, h->f, 0, 1, nl);
	case GDN_CUDA_BF16_STORE:
		return kin_sweeps<__nv_bfloat16, float, float>(h, h->f, 0, 1, nl);
	default:
		return kin_sweeps<double, float, float>(h, h->f, 1, 1, nl);
	}
}

// Sweep-level grouping autotuner: times one transport solve with a launch per
// level and as one cooperative launch over all levels on the handle's own
// buffers (their contents do not change the work; init / set_state rewrite
// them) and keeps the faster.  Cached per (precision, floor(log2 items),
// floor(log2 levels)) for the life of the process.
static std::map<std::pair<int, int>, int> g_tune_kin;

static int autotune_kin(gdn_cuda_handle *h)
{
	int ib = 0, lb = 0;
	const long long nitems = h->ne * h->nv;
	const long long nl = (long long)h->level_off.size() - 1;
	while ((2LL << ib) <= nitems)
		ib++;
	while ((2LL << lb) <= nl)
		lb++;
	const std::pair<int, int> key(h->precision, ib * 64 + lb);
	{
		std::lock_guard<std::mutex> g(g_tune_mu);
		auto it = g_tune_kin.find(key);
		if (it != g_tune_kin.end()) {
			h->kin_mode = it->second;
			return GDN_CUDA_OK;
		}
	}
	GDN_CUDA_TRY(cudaMemsetAsync(h->f, 0, (size_t)60 * nitems * (h->precision == GDN_CUDA_FP32 ? 4 : h->precision == GDN_CUDA_BF16_STORE ? 2 : 8), h->stream));
	GDN_CUDA_TRY(cudaMemsetAsync(h->bt, 0, (size_t)36 * h->nv * (h->nbf > 0 ? h->nbf : 1) * sizeof(double), h->stream));
	// each mode: one warm-up solve, then the best of three solves timed one by
	// one (a solve is well under a millisecond on small meshes, where the
	// modes are within a few per cent of each other)
	cudaEvent_t ev[4];
	for (int i = 0; i < 4; i++)
		GDN_CUDA_TRY(cudaEventCreate(&ev[i]));
	float best = 0.f;
	int pick = 1, rc = GDN_CUDA_OK;
	for (int mode = 1; mode <= 4 && rc == GDN_CUDA_OK; mode++) {
		h->kin_mode = mode;
		long long nlaunch = 0;
		rc = kin_first_sweep(h, nlaunch); // warm-up
		for (int rep = 0; rep < 3 && rc == GDN_CUDA_OK; rep++) {
			cudaEventRecord(ev[rep], h->stream);
			rc = kin_first_sweep(h, nlaunch);
		}
		h->launches += nlaunch;
		if (rc != GDN_CUDA_OK)
			break;
		cudaEventRecord(ev[3], h->stream);
		cudaError_t e = cudaEventSynchronize(ev[3]);
		float ms = 0.f;
		for (int rep = 0; rep < 3 && e == cudaSuccess; rep++) {
			float m = 0.f;
			e = cudaEventElapsedTime(&m, ev[rep], ev[rep + 1]);
			ms = rep == 0 || m < ms ? m : ms;
		}
		if (e != cudaSuccess)
			rc = gdn_cuda_fail(e, "autotune_kin", __FILE__, __LINE__);
		if (mode == 1 || ms < best) {
			best = ms;
			pick = mode;
		}
	}
	for (int i = 0; i < 4; i++)
		cudaEventDestroy(ev[i]);
	if (rc != GDN_CUDA_OK)
		return rc;
	h->kin_mode = pick;
	std::lock_guard<std::mutex> g(g_tune_mu);
	g_tune_kin[key] = pick;
	return GDN_CUDA_OK;
}

// A cooperative sweep whose bounded barrier wait gave up leaves *err set: the
// state is invalid; report it (and clear the flag) at the next synchronising
// call.
static int check_device_error(gdn_cuda_handle *h)
{
	if (!h->err)
		return GDN_CUDA_OK;
	int e = 0;
	GDN_CUDA_TRY(cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	if (e) {
		GDN_CUDA_TRY(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream));
		if (h->bar)
			GDN_CUDA_TRY(cudaMemsetAsync(h->bar, 0, 2 * sizeof(unsigned), h->stream));
		GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
		return gdn_set_error(GDN_CUDA_ERR_TIMEOUT, "kinetic sweep: a grid barrier wait timed out; the state is invalid");
	}
	return GDN_CUDA_OK;
}

static int enqueue_steps(gdn_cuda_handle *h, int nsteps, int &cur, long long &nlaunch)
{
	for (int n = 0; n < nsteps; n++) {
		if (h->scheme == GDN_CUDA_SCHEME_RK3) {
			if (h->precision == GDN_CUDA_FP64)
				GDN_TRY(rk3_enqueue<double>(h, cur, nlaunch));
			else
				GDN_TRY(rk3_enqueue<float>(h, cur, nlaunch));
		} else {
			GDN_TRY(kin_enqueue(h, nlaunch));
		}
	}
	return GDN_CUDA_OK;
}

// host mirror of the device times, as the reference accumulates them
static void bookkeep_step(gdn_cuda_handle *h)
{
	for (int i = 0; i < h->ninst; i++) {
		h->ht_bdof[i] = h->ht[i] + RK_C[2] * h->hdt[i];
		h->ht[i] += h->hdt[i];
	}
	h->steps++;
}

// Step loops as CUDA graphs: RK3 captures 2 steps (6 stages: the ping-pong
// buffers come back to the same parity), one graph per starting parity; the
// level-launch kinetic step captures 1 step.  Everything a step reads that
// changes from step to step (the time) lives on the device.
static int capture_graph(gdn_cuda_handle *h, int key, int unit)
{
	cudaGraph_t graph = nullptr;
	GDN_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
	int cur = key;
	long long nl = 0;
	int rc = enqueue_steps(h, unit, cur, nl);
	cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
	if (rc != GDN_CUDA_OK)
		return rc;
	if (ce != cudaSuccess)
		return gdn_cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
	ce = cudaGraphInstantiate(&h->graph_exec[key], graph, 0);
	cudaGraphDestroy(graph);
	if (ce != cudaSuccess)
		return gdn_cuda_fail(ce, "cudaGraphInstantiate", __FILE__, __LINE__);
	h->graph_nodes[key] = nl;
	return GDN_CUDA_OK;
}

static int advance_impl(gdn_cuda_handle *h, int nsteps)
{
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	const bool graphable = h->use_graph != 0;
	const int unit = h->scheme == GDN_CUDA_SCHEME_RK3 ? 2 : 1;
	while (graphable && nsteps >= unit) {
		const int key = h->scheme == GDN_CUDA_SCHEME_RK3 ? h->cur : 0;
		if (!h->graph_exec[key])
			GDN_TRY(capture_graph(h, key, unit));
		GDN_CUDA_TRY(cudaGraphLaunch(h->graph_exec[key], h->stream));
		for (int u = 0; u < unit; u++)
			bookkeep_step(h);
		h->launches += h->graph_nodes[key];
		nsteps -= unit;
	}
	while (nsteps > 0) {
		long long nl = 0;
		GDN_TRY(enqueue_steps(h, 1, h->cur, nl));
		h->launches += nl;
		bookkeep_step(h);
		nsteps--;
	}
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_advance(gdn_cuda_handle *h, int nsteps)
{
	if (!h || nsteps < 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "advance: bad arguments");
	return advance_impl(h, nsteps);
}

// storage type of the kinetic distributions: 0 FP64, 1 FP32, 2 BF16
static int kin_state_kind(const gdn_cuda_handle *h)
{
	if (h->precision == GDN_CUDA_FP32)
		return 1;
	if (h->precision == GDN_CUDA_BF16_STORE)
		return 2;
	return 0;
}

// kinetic state of instance i <-> its reference layout in the staging buffer
static int kin_pack(gdn_cuda_handle *h, int i, int to_ref)
{
	const int sk = kin_state_kind(h);
	const long long e0 = h->e_off[i], ne = h->e_off[i + 1] - e0;
	const int *pos = h->pos + e0 * h->nv;
	double *st = h->staging + h->w_off[i];
	const long long neq = h->neq_i[i];
	if (sk == 0)
		return launch_kin_pack<double>(as<double>(h->f), pos, ne, h->nv, neq, st, to_ref, h->stream);
	if (sk == 1)
		return launch_kin_pack<float>(as<float>(h->f), pos, ne, h->nv, neq, st, to_ref, h->stream);
	return launch_kin_pack<__nv_bfloat16>(as<__nv_bfloat16>(h->f), pos, ne, h->nv, neq, st, to_ref, h->stream);
}

// dg_init_sol_macro (dg.c:32-59) of every instance with its own data
extern "C" int gdn_cuda_init(gdn_cuda_handle *h)
{
	if (!h)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "init: NULL handle");
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	cudaStream_t s = h->stream;
	const int sk = h->scheme == GDN_CUDA_SCHEME_KINETIC ? kin_state_kind(h) : 0;
	for (int i = 0; i < h->ninst; i++) {
		const long long e0 = h->e_off[i], ne = h->e_off[i + 1] - e0;
		const int *e2q = h->e2q + 10 * e0;
		const Data &d = h->hdata[i];
		if (h->scheme == GDN_CUDA_SCHEME_RK3) {
			if (h->precision == GDN_CUDA_FP64)
				GDN_TRY(launch_init_rk3<double>(e2q, h->node, ne, e0, d, as<double>(h->w[0]), s));
			else
				GDN_TRY(launch_init_rk3<float>(e2q, h->node, ne, e0, d, as<float>(h->w[0]), s));
		} else {
			const int *pos = h->pos + e0 * h->nv;
			if (sk == 0)
				GDN_TRY(launch_init_kin<double>(e2q, h->node, ne, d, h->km, pos, as<double>(h->f), s));
			else if (sk == 1)
				GDN_TRY(launch_init_kin<float>(e2q, h->node, ne, d, h->km, pos, as<float>(h->f), s));
			else
				GDN_TRY(launch_init_kin<__nv_bfloat16>(e2q, h->node, ne, d, h->km, pos, as<__nv_bfloat16>(h->f), s));
		}
		h->launches++;
	}
	if (h->scheme == GDN_CUDA_SCHEME_RK3) {
		h->cur = 0;
		GDN_CUDA_TRY(cudaMemsetAsync(h->k2, 0, 60 * 32 * ((h->ne + 31) / 32) * h->ssize, s));
	}
	GDN_TRY(launch_set_time(h->batch(), 0.0, s));
	h->launches++;
	h->ht.assign(h->ninst, 0.0);
	h->ht_bdof.assign(h->ninst, 0.0);
	h->steps = 0;
	return GDN_CUDA_OK;
}

// reference-layout state -> device (boundary dofs are not state on the
// device: they are analytic data, re-derived when written back).  A batch
// state is the concatenation of the instances' reference-layout vectors.
extern "C" int gdn_cuda_set_state(gdn_cuda_handle *h, const double *wn, double t)
{
	if (!h || !wn)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "set_state: bad arguments");
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	cudaStream_t s = h->stream;
	if (h->scheme == GDN_CUDA_SCHEME_RK3) {
		h->cur = 0;
		for (int i = 0; i < h->ninst; i++) {
			const long long e0 = h->e_off[i], ne = h->e_off[i + 1] - e0;
			const double *src = wn + h->w_off[i];
			double *st = h->staging + h->w_off[i];
			GDN_CUDA_TRY(cudaMemcpyAsync(st, src, 60 * ne * sizeof(double), cudaMemcpyHostToDevice, s));
			if (h->precision == GDN_CUDA_FP64)
				GDN_TRY(launch_rk3_to_tiles<double>(st, as<double>(h->w[0]), e0, ne, s));
			else
				GDN_TRY(launch_rk3_to_tiles<float>(st, as<float>(h->w[0]), e0, ne, s));
			h->launches++;
		}
		GDN_CUDA_TRY(cudaMemsetAsync(h->k2, 0, 60 * 32 * ((h->ne + 31) / 32) * h->ssize, s));
	} else {
		GDN_CUDA_TRY(cudaMemcpyAsync(h->staging, wn, h->w_off.back() * sizeof(double), cudaMemcpyHostToDevice, s));
		for (int i = 0; i < h->ninst; i++) {
			GDN_TRY(kin_pack(h, i, 0));
			h->launches++;
		}
	}
	GDN_TRY(launch_set_time(h->batch(), t, s));
	h->launches++;
	h->ht.assign(h->ninst, t);
	h->ht_bdof.assign(h->ninst, t);
	return GDN_CUDA_OK;
}

static int get_state_impl(gdn_cuda_handle *h, double *wn)
{
	GDN_TRY(check_device_error(h));
	cudaStream_t s = h->stream;
	for (int i = 0; i < h->ninst; i++) {
		const long long e0 = h->e_off[i], ne = h->e_off[i + 1] - e0;
		const long long b0 = h->bf_off[i], nbf = h->bf_off[i + 1] - b0;
		const long long neq = h->neq_i[i];
		double *st = h->staging + h->w_off[i];
		double *dst = wn + h->w_off[i];
		if (h->scheme == GDN_CUDA_SCHEME_RK3) {
			// boundary dofs at the time of the last stage's boundary data
			GDN_TRY(launch_boundary_dofs(h->bxyz + 18 * b0, nbf, h->hdata[i], h->ht_bdof[i], 0, h->km, neq,
										 st + 60 * ne, s));
			h->launches++;
			if (h->precision == GDN_CUDA_FP64)
				GDN_TRY(launch_rk3_from_tiles<double>(as<double>(h->w[h->cur]), st, e0, ne, s));
			else
				GDN_TRY(launch_rk3_from_tiles<float>(as<float>(h->w[h->cur]), st, e0, ne, s));
			h->launches++;
			GDN_CUDA_TRY(cudaMemcpyAsync(dst, st, 60 * ne * sizeof(double), cudaMemcpyDeviceToHost, s));
			if (nbf > 0)
				GDN_CUDA_TRY(cudaMemcpyAsync(dst + 60 * ne, st + 60 * ne, 36 * nbf * sizeof(double),
											 cudaMemcpyDeviceToHost, s));
		} else {
			// boundary dofs after dg_update_boundary(simu, t) (relaxation.c:175)
			GDN_TRY(launch_boundary_dofs(h->bxyz + 18 * b0, nbf, h->hdata[i], h->ht[i], 1, h->km, neq, st + 10 * ne,
										 s));
			GDN_TRY(kin_pack(h, i, 1));
			h->launches += 2;
		}
	}
	if (h->scheme == GDN_CUDA_SCHEME_KINETIC)
		GDN_CUDA_TRY(cudaMemcpyAsync(wn, h->staging, h->w_off.back() * sizeof(double), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_get_state(gdn_cuda_handle *h, double *wn)
{
	if (!h || !wn)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "get_state: bad arguments");
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	return get_state_impl(h, wn);
}

extern "C" int gdn_cuda_step_host(gdn_cuda_handle *h, double *wn, int nsteps)
{
	if (!h || !wn || nsteps < 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "step_host: bad arguments");
	if (h->ninst > 1)
		return gdn_set_error(GDN_CUDA_ERR_UNSUPPORTED, "step_host: one instance per handle");
	GDN_TRY(gdn_cuda_set_state(h, wn, h->ht[0]));
	GDN_TRY(advance_impl(h, nsteps));
	return get_state_impl(h, wn);
}

extern "C" int gdn_cuda_solve(gdn_cuda_handle *h, int itermax, double *wn, double *t, double *cpu_running_t)
{
	if (!h || !wn || itermax < 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "solve: bad arguments");
	GDN_TRY(gdn_cuda_init(h));
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	auto t0 = std::chrono::steady_clock::now();
	GDN_TRY(advance_impl(h, itermax));
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	auto t1 = std::chrono::steady_clock::now();
	GDN_TRY(get_state_impl(h, wn));
	if (t)
		*t = h->ht[0];
	if (cpu_running_t)
		*cpu_running_t = std::chrono::duration<double>(t1 - t0).count();
	return GDN_CUDA_OK;
}

// simulation_error_l2 of instance i at its current time
static int error_l2_impl(gdn_cuda_handle *h, int i, double *err)
{
	GDN_TRY(check_device_error(h));
	cudaStream_t s = h->stream;
	const bool kin = h->scheme == GDN_CUDA_SCHEME_KINETIC;
	const int sk = kin ? kin_state_kind(h) : (h->precision == GDN_CUDA_FP64 ? 0 : 1);
	const long long e0 = h->e_off[i], ne = h->e_off[i + 1] - e0;
	const long long te0 = kin ? 0 : e0; // RK3: tiled state indexed by global element; kinetic: through pos
	const int *pos = kin ? h->pos + e0 * h->nv : nullptr;
	const int *e2q = h->e2q + 10 * e0;
	const double *geom = h->geom64 + 10 * e0;
	void *st = kin ? h->f : h->w[h->cur];
	const double t = h->ht[i];
	const Data &d = h->hdata[i];
	if (sk == 0)
		GDN_TRY(launch_error_l2<double>(as<double>(st), kin, te0, h->nv, pos, e2q, h->node, geom, ne, d, t,
										h->partial, h->nblk_err, h->result, s));
	else if (sk == 1)
		GDN_TRY(launch_error_l2<float>(as<float>(st), kin, te0, h->nv, pos, e2q, h->node, geom, ne, d, t, h->partial,
									   h->nblk_err, h->result, s));
	else
		GDN_TRY(launch_error_l2<__nv_bfloat16>(as<__nv_bfloat16>(st), kin, te0, h->nv, pos, e2q, h->node, geom, ne, d,
											   t, h->partial, h->nblk_err, h->result, s));
	h->launches += 2;
	GDN_CUDA_TRY(cudaMemcpyAsync(h->host_result, h->result, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	*err = h->host_result[0];
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_error_l2(gdn_cuda_handle *h, double *err)
{
	if (!h || !err)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "error_l2: bad arguments");
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	return error_l2_impl(h, 0, err);
}

extern "C" int gdn_cuda_error_l2_batch(gdn_cuda_handle *h, double *err)
{
	if (!h || !err)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "error_l2_batch: bad arguments");
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	for (int i = 0; i < h->ninst; i++)
		GDN_TRY(error_l2_impl(h, i, err + i));
	return GDN_CUDA_OK;
}

// ------------------------------------------------------------ output --
// io_save_all (src/io/io_hdf5.c:355-368) with raw little-endian binary files
// in place of HDF5 (libhdf5 is optional for this library): <base>_mesh_conn.bin
// (int32 [ne][10] elem2qnode, instance-local), <base>_mesh_nodes.bin (float64
// [nq][3]), <base>_data_%04d.bin (float64 [m][nq]: component im of node in
// taken at its first element and first local node, io_hdf5.c:179-213), and
// <base>_simulation_%04d.xmf describing them (Tet_10 topology; kinetic: the
// distributions f%d and w%d = sum over velocities).
static int write_file(const std::string &path, const void *data, size_t bytes)
{
	FILE *f = std::fopen(path.c_str(), "wb");
	if (!f)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, ("save_xdmf: cannot open " + path).c_str());
	const size_t w = bytes ? std::fwrite(data, 1, bytes, f) : 0;
	const int closed = std::fclose(f);
	if (w != bytes || closed != 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, ("save_xdmf: cannot write " + path).c_str());
	return GDN_CUDA_OK;
}

static std::string base_name(const std::string &p)
{
	const size_t k = p.find_last_of('/');
	return k == std::string::npos ? p : p.substr(k + 1);
}

extern "C" int gdn_cuda_save_xdmf(gdn_cuda_handle *h, int instance, const char *basename, int iter_id)
{
	if (!h || !basename || instance < 0 || instance >= h->ninst)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "save_xdmf: bad arguments");
	GDN_TRY(check_device_error(h));
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	cudaStream_t s = h->stream;
	const long long e0 = h->e_off[instance], ne = h->e_off[instance + 1] - e0;
	const long long q0 = h->q_off[instance], nq = h->q_off[instance + 1] - q0;
	const bool kin = h->scheme == GDN_CUDA_SCHEME_KINETIC;
	const int m = kin ? 6 * h->nv : 6;
	std::vector<int> conn(10 * ne);
	std::vector<double> nodes(3 * nq), vals((size_t)m * nq);
	int *owner = nullptr;
	double *dv = nullptr;
	cudaError_t ce = cudaMalloc(&owner, (nq > 0 ? nq : 1) * sizeof(int));
	if (ce == cudaSuccess)
		ce = cudaMalloc(&dv, ((size_t)m * nq > 0 ? (size_t)m * nq : 1) * sizeof(double));
	int rc = ce == cudaSuccess ? GDN_CUDA_OK : gdn_cuda_fail(ce, "save_xdmf: cudaMalloc", __FILE__, __LINE__);
	if (rc == GDN_CUDA_OK) {
		const int sk = kin ? kin_state_kind(h) : (h->precision == GDN_CUDA_FP64 ? 0 : 1);
		const void *st = kin ? h->f : h->w[h->cur];
		rc = launch_node_values(st, sk, kin, h->nv, h->pos, h->e2q, e0, ne, q0, nq, owner, dv, s);
		h->launches += 2;
	}
	if (rc == GDN_CUDA_OK) {
		ce = cudaMemcpyAsync(vals.data(), dv, vals.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
		if (ce == cudaSuccess)
			ce = cudaMemcpyAsync(conn.data(), h->e2q + 10 * e0, conn.size() * sizeof(int), cudaMemcpyDeviceToHost, s);
		if (ce == cudaSuccess)
			ce = cudaMemcpyAsync(nodes.data(), h->node + 3 * q0, nodes.size() * sizeof(double), cudaMemcpyDeviceToHost,
								 s);
		if (ce == cudaSuccess)
			ce = cudaStreamSynchronize(s);
		if (ce != cudaSuccess)
			rc = gdn_cuda_fail(ce, "save_xdmf: read-back", __FILE__, __LINE__);
	}
	cudaFree(owner);
	cudaFree(dv);
	if (rc != GDN_CUDA_OK)
		return rc;
	for (auto &q : conn)
		q -= (int)q0;
	char buf[64];
	const std::string base = basename;
	std::snprintf(buf, sizeof(buf), "_data_%04d.bin", iter_id);
	const std::string conn_f = base + "_mesh_conn.bin", node_f = base + "_mesh_nodes.bin", data_f = base + buf;
	std::snprintf(buf, sizeof(buf), "_simulation_%04d.xmf", iter_id);
	const std::string xmf_f = base + buf;
	GDN_TRY(write_file(conn_f, conn.data(), conn.size() * sizeof(int)));
	GDN_TRY(write_file(node_f, nodes.data(), nodes.size() * sizeof(double)));
	GDN_TRY(write_file(data_f, vals.data(), vals.size() * sizeof(double)));
	// data items refer to the binary files by name, next to the .xmf
	const std::string cb = base_name(conn_f), nb = base_name(node_f), db = base_name(data_f);
	std::string x;
	char line[512];
	x += "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n";
	x += "<Xdmf Version=\"2.0\">\n<Domain>\n<Grid Name=\"TheMesh\">\n";
	std::snprintf(line, sizeof(line), "<Time Value=\"%f\"/>\n", h->ht[instance]);
	x += line;
	std::snprintf(line, sizeof(line),
				  "<Topology TopologyType=\"Tet_10\" NumberOfElements=\"%lld\">\n<DataItem Dimensions=\"%lld 10\" "
				  "NumberType=\"Int\" Precision=\"4\" Format=\"Binary\" Endian=\"Little\">%s</DataItem>\n</Topology>\n",
				  ne, ne, cb.c_str());
	x += line;
	std::snprintf(line, sizeof(line),
				  "<Geometry GeometryType=\"XYZ\">\n<DataItem Dimensions=\"%lld 3\" NumberType=\"Float\" Precision=\"8\" "
				  "Format=\"Binary\" Endian=\"Little\">%s</DataItem>\n</Geometry>\n",
				  nq, nb.c_str());
	x += line;
	auto item = [&](int im, const char *indent) {
		std::snprintf(line, sizeof(line),
					  "%s<DataItem Dimensions=\"%lld 1\" NumberType=\"Float\" Precision=\"8\" Format=\"Binary\" "
					  "Endian=\"Little\" Seek=\"%lld\">%s</DataItem>\n",
					  indent, nq, (long long)im * nq * 8, db.c_str());
		x += line;
	};
	const char *prefix = kin ? "f" : "w";
	for (int im = 0; im < m; im++) {
		std::snprintf(line, sizeof(line), "<Attribute Name=\"%s%d\" Center=\"Node\">\n", prefix, im);
		x += line;
		item(im, "");
		x += "</Attribute>\n";
	}
	if (kin) { // macro variables w_iw = sum_iv f_(iw * nb_v + iv)
		for (int iw = 0; iw < 6; iw++) {
			std::snprintf(line, sizeof(line), "<Attribute Name=\"w%d\" Center=\"Node\">\n<DataItem ItemType=\"Function\" Function=\"",
						  iw);
			x += line;
			for (int iv = 0; iv < h->nv; iv++) {
				std::snprintf(line, sizeof(line), "%s$%d", iv ? "+" : "", iv);
				x += line;
			}
			std::snprintf(line, sizeof(line), "\" Dimensions=\"%lld 1\">\n", nq);
			x += line;
			for (int iv = 0; iv < h->nv; iv++)
				item(iw * h->nv + iv, "  ");
			x += "</DataItem>\n</Attribute>\n";
		}
	}
	x += "</Grid>\n</Domain>\n</Xdmf>\n";
	return write_file(xmf_f, x.data(), x.size());
}

// ------------------------------------------------------- convergence --
// New time step of a single-instance RK3 handle: the step graphs hold the
// old one in their kernel parameters and are captured again.
static int rk3_set_dt(gdn_cuda_handle *h, double dt)
{
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	h->hdt.assign(h->ninst, dt);
	GDN_CUDA_TRY(cudaMemcpyAsync(h->dt_dev, h->hdt.data(), h->ninst * sizeof(double), cudaMemcpyHostToDevice,
								 h->stream));
	for (int k = 0; k < 2; k++)
		if (h->graph_exec[k]) {
			cudaGraphExecDestroy(h->graph_exec[k]);
			h->graph_exec[k] = nullptr;
		}
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	return GDN_CUDA_OK;
}

// dg_solve + simulation_error_l2 of one run of a study
static int conv_run(gdn_cuda_handle *h, int iter, double *err)
{
	GDN_TRY(gdn_cuda_init(h));
	GDN_TRY(advance_impl(h, iter));
	return error_l2_impl(h, 0, err);
}

// get_order (src/utils/convergence.c:25-41): log(e_prev / e) / log(x_prev / x)
static double conv_order(double e_prev, double e, double x_prev, double x)
{
	return std::log(e_prev / e) / std::log(x_prev / x);
}

extern "C" int gdn_cuda_time_convergence(const gdn_cuda_mesh *mesh, const gdn_cuda_tables *tables,
										 const gdn_cuda_model *model, const gdn_cuda_data *data,
										 const gdn_cuda_config *config, double init_dt, double tmax, int nb_run,
										 double *dt_out, int *iter_out, double *err_out, double *order_out)
{
	if (nb_run < 1 || !dt_out || !iter_out || !err_out || !order_out || !model || !(init_dt > 0.0) ||
		!std::isfinite(init_dt) || !std::isfinite(tmax))
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "time_convergence: bad arguments");
	// the reference's time grid: init_iter = floor(tmax / dt) - 1 steps, tmax
	// rounded down to a multiple of dt, dt halved and the steps doubled per run
	const int iter0 = (int)std::floor(tmax / init_dt) - 1;
	if (iter0 < 1)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "time_convergence: tmax shorter than two steps");
	const double tmax0 = iter0 * init_dt;
	gdn_cuda_handle *h = nullptr;
	int rc = GDN_CUDA_OK;
	for (int k = 0; k < nb_run && rc == GDN_CUDA_OK; k++) {
		const double dt = k == 0 ? init_dt : 0.5 * dt_out[k - 1];
		const long long want = (long long)iter0 << k;
		const long long iter = (long long)std::floor(tmax0 / dt);
		if (iter != want || iter > 2147483647LL) {
			rc = gdn_set_error(GDN_CUDA_ERR_INVALID, "time_convergence: the halved time grid does not reach tmax");
			break;
		}
		if (h && model->scheme == GDN_CUDA_SCHEME_RK3) {
			rc = rk3_set_dt(h, dt);
		} else {
			if (h)
				gdn_cuda_detach(h);
			h = nullptr;
			rc = gdn_cuda_attach(mesh, tables, model, data, config, dt, &h);
		}
		if (rc == GDN_CUDA_OK)
			rc = conv_run(h, (int)iter, &err_out[k]);
		dt_out[k] = dt;
		iter_out[k] = (int)iter;
		order_out[k] = k == 0 ? -1.0 : conv_order(err_out[k - 1], err_out[k], dt_out[k - 1], dt);
	}
	if (h) {
		std::string msg = g_last_error;
		gdn_cuda_detach(h);
		g_last_error = msg;
	}
	return rc;
}

extern "C" int gdn_cuda_space_convergence(const gdn_cuda_mesh *const *meshes, int nb_run,
										  const gdn_cuda_tables *tables, const gdn_cuda_model *model,
										  const gdn_cuda_data *data, const gdn_cuda_config *config, double init_dt,
										  double tmax, int time_refinement, double *dt_out, int *iter_out,
										  double *hmin_out, double *err_out, double *order_out)
{
	if (!meshes || nb_run < 1 || !dt_out || !iter_out || !hmin_out || !err_out || !order_out || !model ||
		!(init_dt > 0.0) || !std::isfinite(init_dt) || !std::isfinite(tmax))
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "space_convergence: bad arguments");
	const int iter0 = (int)std::floor(tmax / init_dt) - 1;
	if (iter0 < 1)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "space_convergence: tmax shorter than two steps");
	const double tmax0 = iter0 * init_dt;
	for (int k = 0; k < nb_run; k++) {
		const double dt = k == 0 || !time_refinement ? init_dt : 0.5 * dt_out[k - 1];
		const long long want = time_refinement ? (long long)iter0 << k : iter0;
		const long long iter = (long long)std::floor(tmax0 / dt);
		if (iter != want || iter > 2147483647LL)
			return gdn_set_error(GDN_CUDA_ERR_INVALID, "space_convergence: the time grid does not reach tmax");
		GDN_TRY(gdn_cuda_mesh_hmin(meshes[k], &hmin_out[k]));
		// the reference asserts meshes refined by 2 (convergence.c:157)
		if (k > 0 && !(std::fabs(hmin_out[k - 1] / hmin_out[k] - 2.0) < 1e-6))
			return gdn_set_error(GDN_CUDA_ERR_INVALID, "space_convergence: consecutive meshes must halve hmin");
		gdn_cuda_handle *h = nullptr;
		GDN_TRY(gdn_cuda_attach(meshes[k], tables, model, data, config, dt, &h));
		const int rc = conv_run(h, (int)iter, &err_out[k]);
		std::string msg = g_last_error;
		gdn_cuda_detach(h);
		g_last_error = msg;
		if (rc != GDN_CUDA_OK)
			return rc;
		dt_out[k] = dt;
		iter_out[k] = (int)iter;
		order_out[k] = k == 0 ? -1.0 : conv_order(err_out[k - 1], err_out[k], hmin_out[k - 1], hmin_out[k]);
	}
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_set_wait_limit(gdn_cuda_handle *h, long long polls)
{
	if (!h || polls < 0)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "set_wait_limit: bad arguments");
	GDN_CUDA_TRY(cudaSetDevice(h->device));
	GDN_CUDA_TRY(cudaStreamSynchronize(h->stream));
	h->spin_limit = polls;
	// the limit is a kernel parameter of the captured step loops
	for (int k = 0; k < 2; k++)
		if (h->graph_exec[k]) {
			cudaGraphExecDestroy(h->graph_exec[k]);
			h->graph_exec[k] = nullptr;
		}
	return GDN_CUDA_OK;
}

// ------------------------------------------------------ data check --
extern "C" int gdn_cuda_eval_data(const gdn_cuda_data *d, long long npts, const double *xyz, double t, double *w,
								  int device)
{
	if (!d || npts < 0 || (npts > 0 && (!xyz || !w)))
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "eval_data: bad arguments");
	GDN_TRY(validate_data(d));
	if (npts == 0)
		return GDN_CUDA_OK;
	GDN_CUDA_TRY(cudaSetDevice(device));
	cudaStream_t s = nullptr;
	double *xd = nullptr, *wd = nullptr;
	int rc = GDN_CUDA_OK;
	cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
	if (e == cudaSuccess)
		e = cudaMalloc(&xd, (size_t)npts * 3 * sizeof(double));
	if (e == cudaSuccess)
		e = cudaMalloc(&wd, (size_t)npts * 6 * sizeof(double));
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(xd, xyz, (size_t)npts * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
	if (e == cudaSuccess) {
		rc = launch_eval_data(xd, npts, to_data(d), t, wd, s);
		if (rc == GDN_CUDA_OK)
			e = cudaMemcpyAsync(w, wd, (size_t)npts * 6 * sizeof(double), cudaMemcpyDeviceToHost, s);
	}
	if (e == cudaSuccess && rc == GDN_CUDA_OK)
		e = cudaStreamSynchronize(s);
	if (e != cudaSuccess && rc == GDN_CUDA_OK)
		rc = e == cudaErrorMemoryAllocation ? gdn_set_error(GDN_CUDA_ERR_OOM, "eval_data: device allocation failed")
											: gdn_cuda_fail(e, "eval_data", __FILE__, __LINE__);
	cudaFree(xd);
	cudaFree(wd);
	if (s)
		cudaStreamDestroy(s);
	return rc;
}

extern "C" int gdn_cuda_get_time(gdn_cuda_handle *h, double *t)
{
	if (!h || !t)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "get_time: bad arguments");
	*t = h->ht[0];
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_kin_sweep_mode(gdn_cuda_handle *h, int *mode)
{
	if (!h || !mode)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "kin_sweep_mode: bad arguments");
	*mode = h->scheme == GDN_CUDA_SCHEME_KINETIC ? h->kin_mode : 0;
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_rk3_variant(gdn_cuda_handle *h, int *variant, int *min_ctas_per_sm)
{
	if (!h || !variant)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "rk3_variant: bad arguments");
	const bool rk = h->scheme == GDN_CUDA_SCHEME_RK3;
	*variant = rk ? h->rk3_variant + 1 : 0;
	if (min_ctas_per_sm)
		*min_ctas_per_sm = rk ? rk3_min_blocks(h->precision == GDN_CUDA_FP64, h->rk3_variant) : 0;
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_num_instances(gdn_cuda_handle *h, int *n)
{
	if (!h || !n)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "num_instances: bad arguments");
	*n = h->ninst;
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_instance_info(gdn_cuda_handle *h, int i, double *t, long long *nbelems,
									  long long *w_offset, long long *wlen)
{
	if (!h || i < 0 || i >= h->ninst)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "instance_info: bad arguments");
	if (t)
		*t = h->ht[i];
	if (nbelems)
		*nbelems = h->e_off[i + 1] - h->e_off[i];
	if (w_offset)
		*w_offset = h->w_off[i];
	if (wlen)
		*wlen = h->w_off[i + 1] - h->w_off[i];
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_state_size(gdn_cuda_handle *h, long long *wlen)
{
	if (!h || !wlen)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "state_size: bad arguments");
	*wlen = h->w_off.back();
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_num_levels(gdn_cuda_handle *h, int *nlevels)
{
	if (!h || !nlevels)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "num_levels: bad arguments");
	*nlevels = h->scheme == GDN_CUDA_SCHEME_KINETIC ? (int)h->level_off.size() - 1 : 0;
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_launch_count(gdn_cuda_handle *h, long long *count)
{
	if (!h || !count)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "launch_count: bad arguments");
	*count = h->launches;
	return GDN_CUDA_OK;
}

extern "C" int gdn_cuda_stream(gdn_cuda_handle *h, void **stream)
{
	if (!h || !stream)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "stream: bad arguments");
	*stream = (void *)h->stream;
	return GDN_CUDA_OK;
}
