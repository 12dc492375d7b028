// gdn_cuda_mesh_build_gpu: the connectivity arrays of gdn_cuda_mesh_build
// (the reference's mesh_build_connectivity, src/mesh/mesh.c:803-1268 and
// 1234-1268), built on the device with the same numbering, bit for bit:
//   faces      4 ne sorted vertex triples, ordered lexicographically with the
//              element index as the tie-break (two stable radix sorts: the
//              (v1, v2) pair, then v0); equal neighbours in that order are
//              the two sides of an interior face;
//   face list  (element, local face) in order, kept when the neighbour index
//              is below the element's (L = the larger index), numbered by a
//              prefix sum; boundary faces numbered the same way;
//   P2 nodes   used vertices in vertex order, then the edges in ascending
//              (min, max) vertex order (a stable sort of the 6 ne edge keys
//              and a prefix sum over the runs of equal keys).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <vector>

#include "aux.h"
#include "kernels.h"

namespace gdn {

__constant__ int c_t4face[4][3] = {{0, 3, 2}, {0, 1, 3}, {0, 2, 1}, {1, 2, 3}};
__constant__ int c_t4edge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
__constant__ int c_f2n[4][6] = {{0, 3, 2, 7, 9, 6}, {0, 1, 3, 4, 8, 7}, {0, 2, 1, 6, 5, 4}, {1, 2, 3, 5, 9, 8}};

__global__ void mb_face_keys(const int *__restrict__ e2n, long long ne, unsigned long long *k12, int *k0, int *idx)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= 4 * ne)
		return;
	const long long ie = u >> 2;
	const int f = (int)(u & 3);
	int a = e2n[4 * ie + c_t4face[f][0]], b = e2n[4 * ie + c_t4face[f][1]], c = e2n[4 * ie + c_t4face[f][2]];
	int t;
	if (a > b) t = a, a = b, b = t;
	if (b > c) t = b, b = c, c = t;
	if (a > b) t = a, a = b, b = t;
	k12[u] = ((unsigned long long)(unsigned)b << 32) | (unsigned)c;
	k0[u] = a;
	idx[u] = (int)u;
}

// sorted faces: v0 = k0s[i], (v1, v2) = k12 of face fidx[i]
__global__ void mb_pair_faces(const int *__restrict__ k0s, const int *__restrict__ fidx,
							  const unsigned long long *__restrict__ k12, long long n, int *e2e, int *bad)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i + 1 >= n)
		return;
	const int fa = fidx[i], fb = fidx[i + 1];
	if (k0s[i] != k0s[i + 1] || k12[fa] != k12[fb])
		return;
	// first of a run of equal keys only
	if (i > 0 && k0s[i - 1] == k0s[i] && k12[fidx[i - 1]] == k12[fa])
		return;
	if (i + 2 < n && k0s[i + 2] == k0s[i] && k12[fidx[i + 2]] == k12[fa]) {
		atomicExch(bad, 1); // non-manifold
		return;
	}
	e2e[fa] = fb >> 2;
	e2e[fb] = fa >> 2;
}

__global__ void mb_face_flags(const int *__restrict__ e2e, long long ne, int *keep, int *bkeep)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= 4 * ne)
		return;
	const int ie2 = e2e[u];
	const int k = ie2 < (int)(u >> 2);
	keep[u] = k;
	bkeep[u] = k && ie2 < 0;
}

__global__ void mb_vertex_used(const int *__restrict__ e2n, long long n4, int *used)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u < n4)
		used[e2n[u]] = 1;
}

__global__ void mb_edge_keys(const int *__restrict__ e2n, long long ne, unsigned long long *key, int *idx)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= 6 * ne)
		return;
	const long long ie = u / 6;
	const int e = (int)(u % 6);
	unsigned a = (unsigned)e2n[4 * ie + c_t4edge[e][0]], b = (unsigned)e2n[4 * ie + c_t4edge[e][1]];
	if (a > b) {
		const unsigned t = a;
		a = b;
		b = t;
	}
	key[u] = ((unsigned long long)a << 32) | b;
	idx[u] = (int)u;
}

__global__ void mb_edge_heads(const unsigned long long *__restrict__ ks, long long n, int *head)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i < n)
		head[i] = (i == 0 || ks[i] != ks[i - 1]) ? 1 : 0;
}

// elem2qnode edge entries and edge-node coordinates (0.5 a + 0.5 b)
__global__ void mb_edge_nodes(const unsigned long long *__restrict__ ks, const int *__restrict__ eidx,
							  const int *__restrict__ head, const int *__restrict__ run, long long n, int nvq,
							  const double *__restrict__ coords, int *e2q, double *node)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int q = nvq + run[i] + head[i] - 1; // inclusive run index
	const long long u = eidx[i];
	e2q[10 * (u / 6) + 4 + (u % 6)] = q;
	if (head[i]) {
		const long long a = (long long)(ks[i] >> 32), b = (long long)(ks[i] & 0xffffffffull);
		for (int c = 0; c < 3; c++)
			node[3LL * q + c] = 0.5 * coords[3 * a + c] + 0.5 * coords[3 * b + c];
	}
}

__global__ void mb_vertex_nodes(const int *__restrict__ used, const int *__restrict__ vmap, int nbnodes,
								const double *__restrict__ coords, double *node)
{
	const int v = blockIdx.x * blockDim.x + threadIdx.x;
	if (v < nbnodes && used[v])
		for (int c = 0; c < 3; c++)
			node[3LL * vmap[v] + c] = coords[3LL * v + c];
}

__global__ void mb_vertex_e2q(const int *__restrict__ e2n, const int *__restrict__ vmap, long long ne, int *e2q)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u < 4 * ne)
		e2q[10 * (u >> 2) + (u & 3)] = vmap[e2n[u]];
}

__global__ void mb_faces(const int *__restrict__ e2e, const int *__restrict__ keep, const int *__restrict__ fpos,
						 const int *__restrict__ bpos, long long ne, int *e2q, int *face2elem, int *fnode2enode,
						 int *boundaryface, int *bad)
{
	const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (u >= 4 * ne || !keep[u])
		return;
	const long long ie = u >> 2;
	const int f = (int)(u & 3);
	const int ie2 = e2e[u];
	const long long fc = fpos[u];
	face2elem[4 * fc + 0] = (int)ie;
	face2elem[4 * fc + 1] = f;
	face2elem[4 * fc + 2] = ie2;
	face2elem[4 * fc + 3] = -1;
	if (ie2 >= 0)
		for (int f2 = 0; f2 < 4; f2++)
			if (e2e[4LL * ie2 + f2] == (int)ie) {
				face2elem[4 * fc + 3] = f2;
				break;
			}
	const long long bc = bpos[u];
	for (int j = 0; j < 6; j++) {
		const int inoe = c_f2n[f][j];
		fnode2enode[12 * fc + j] = inoe;
		const int gq = e2q[10 * ie + inoe];
		if (ie2 < 0) {
			fnode2enode[12 * fc + 6 + j] = j;
			e2q[10 * ne + 6 * bc + j] = gq;
		} else {
			int r = 0;
			while (r < 10 && e2q[10LL * ie2 + r] != gq)
				r++;
			if (r == 10) {
				atomicExch(bad, 2);
				r = 0;
			}
			fnode2enode[12 * fc + 6 + j] = r;
		}
	}
	if (ie2 < 0)
		boundaryface[bc] = (int)fc;
}

__global__ void mb_gather(const int *__restrict__ src, const int *__restrict__ order, long long n, int *out)
{
	const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = src[order[i]];
}

} // namespace gdn

// Device buffers of one build, freed on every exit.
namespace {
struct MbBufs {
	std::vector<void *> p;
	template <typename X>
	cudaError_t get(X **out, size_t n)
	{
		void *q = nullptr;
		cudaError_t e = cudaMalloc(&q, (n > 0 ? n : 1) * sizeof(X));
		if (e == cudaSuccess)
			p.push_back(q);
		*out = reinterpret_cast<X *>(q);
		return e;
	}
	~MbBufs()
	{
		for (void *q : p)
			cudaFree(q);
	}
};
struct StreamGuard {
	cudaStream_t s = nullptr;
	~StreamGuard()
	{
		if (s)
			cudaStreamDestroy(s);
	}
};
// last element of an exclusive scan plus the last flag: the total
int scan_total(const int *scan, const int *flag, long long n, cudaStream_t s, int *out)
{
	int a = 0, b = 0;
	GDN_CUDA_TRY(cudaMemcpyAsync(&a, scan + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(&b, flag + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	*out = a + b;
	return GDN_CUDA_OK;
}
} // namespace

extern "C" int gdn_cuda_mesh_build_gpu(int nbnodes, const double *coords, int nbelems, const int *elem2node,
									   int *nbfaces_out, int *nbf_out, int *nbq_out, int *face2elem,
									   int *fnode2enode, int *boundaryface, int *elem2qnode, double *node, int device)
{
	using namespace gdn;
	if (nbnodes <= 0 || nbelems <= 0 || !coords || !elem2node || !nbfaces_out || !nbf_out || !nbq_out)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "mesh_build_gpu: bad arguments");
	const long long ne = nbelems;
	if (6 * ne > 0x7fffffffLL)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "mesh_build_gpu: too many elements for 32-bit indices");
	for (long long i = 0; i < 4 * ne; i++)
		if (elem2node[i] < 0 || elem2node[i] >= nbnodes)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "mesh_build_gpu: elem2node index out of range");
	GDN_CUDA_TRY(cudaSetDevice(device));
	StreamGuard sg;
	GDN_CUDA_TRY(cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking));
	const cudaStream_t s = sg.s;
	MbBufs B;
	const long long nfk = 4 * ne, nek = 6 * ne;
	int *e2n, *k0, *k0g, *k0s, *idx, *fidx1, *fidx, *e2e, *keep, *bkeep, *fpos, *bpos, *bad, *used, *vmap, *eidx,
		*eidxs, *head, *run;
	unsigned long long *k12, *k12s, *ek, *eks;
	double *crd;
	GDN_CUDA_TRY(B.get(&e2n, nfk));
	GDN_CUDA_TRY(B.get(&crd, 3LL * nbnodes));
	GDN_CUDA_TRY(B.get(&k0, nfk));
	GDN_CUDA_TRY(B.get(&k0g, nfk));
	GDN_CUDA_TRY(B.get(&k0s, nfk));
	GDN_CUDA_TRY(B.get(&idx, nfk));
	GDN_CUDA_TRY(B.get(&fidx1, nfk));
	GDN_CUDA_TRY(B.get(&fidx, nfk));
	GDN_CUDA_TRY(B.get(&k12, nfk));
	GDN_CUDA_TRY(B.get(&k12s, nfk));
	GDN_CUDA_TRY(B.get(&e2e, nfk));
	GDN_CUDA_TRY(B.get(&keep, nfk));
	GDN_CUDA_TRY(B.get(&bkeep, nfk));
	GDN_CUDA_TRY(B.get(&fpos, nfk));
	GDN_CUDA_TRY(B.get(&bpos, nfk));
	GDN_CUDA_TRY(B.get(&bad, 1));
	GDN_CUDA_TRY(B.get(&used, nbnodes));
	GDN_CUDA_TRY(B.get(&vmap, nbnodes));
	GDN_CUDA_TRY(B.get(&ek, nek));
	GDN_CUDA_TRY(B.get(&eks, nek));
	GDN_CUDA_TRY(B.get(&eidx, nek));
	GDN_CUDA_TRY(B.get(&eidxs, nek));
	GDN_CUDA_TRY(B.get(&head, nek));
	GDN_CUDA_TRY(B.get(&run, nek));
	GDN_CUDA_TRY(cudaMemcpyAsync(e2n, elem2node, nfk * sizeof(int), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(crd, coords, 3LL * nbnodes * sizeof(double), cudaMemcpyHostToDevice, s));
	GDN_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
	GDN_CUDA_TRY(cudaMemsetAsync(e2e, 0xff, nfk * sizeof(int), s)); // -1: no neighbour
	GDN_CUDA_TRY(cudaMemsetAsync(used, 0, nbnodes * sizeof(int), s));
	const unsigned gf = (unsigned)((nfk + 255) / 256), ge = (unsigned)((nek + 255) / 256),
				   gv = (unsigned)((nbnodes + 255) / 256);
	// scratch of the largest CUB call
	size_t tmp_bytes = 0, need = 0;
	GDN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, k12, k12s, idx, fidx1, (int)nfk, 0, 64, s));
	tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
	GDN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, k0g, k0s, fidx1, fidx, (int)nfk, 0, 32, s));
	tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
	GDN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, ek, eks, eidx, eidxs, (int)nek, 0, 64, s));
	tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
	GDN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, need, keep, fpos, (int)nek, s));
	tmp_bytes = need > tmp_bytes ? need : tmp_bytes;
	char *tmp;
	GDN_CUDA_TRY(B.get(&tmp, tmp_bytes));

	// faces in lexicographic (v0, v1, v2, element) order: stable sort by
	// (v1, v2), then stable sort by v0
	mb_face_keys<<<gf, 256, 0, s>>>(e2n, ne, k12, k0, idx);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k12, k12s, idx, fidx1, (int)nfk, 0, 64, s));
	mb_gather<<<gf, 256, 0, s>>>(k0, fidx1, nfk, k0g);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k0g, k0s, fidx1, fidx, (int)nfk, 0, 32, s));
	mb_pair_faces<<<gf, 256, 0, s>>>(k0s, fidx, k12, nfk, e2e, bad);
	GDN_CUDA_TRY(cudaGetLastError());
	mb_face_flags<<<gf, 256, 0, s>>>(e2e, ne, keep, bkeep);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, keep, fpos, (int)nfk, s));
	GDN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, bkeep, bpos, (int)nfk, s));
	// P2 nodes: used vertices in vertex order, then edges in key order
	mb_vertex_used<<<gf, 256, 0, s>>>(e2n, nfk, used);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, used, vmap, nbnodes, s));
	mb_edge_keys<<<ge, 256, 0, s>>>(e2n, ne, ek, eidx);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, ek, eks, eidx, eidxs, (int)nek, 0, 64, s));
	mb_edge_heads<<<ge, 256, 0, s>>>(eks, nek, head);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, head, run, (int)nek, s));

	int nf = 0, nbf = 0, nvq = 0, nedge = 0, hbad = 0;
	GDN_TRY(scan_total(fpos, keep, nfk, s, &nf));
	GDN_TRY(scan_total(bpos, bkeep, nfk, s, &nbf));
	GDN_TRY(scan_total(vmap, used, nbnodes, s, &nvq));
	GDN_TRY(scan_total(run, head, nek, s, &nedge));
	GDN_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	if (hbad)
		return gdn_set_error(GDN_CUDA_ERR_MESH, "mesh_build_gpu: non-manifold face");
	const long long nq = (long long)nvq + nedge;
	if (nq > 0x7fffffffLL)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "mesh_build_gpu: too many P2 nodes for 32-bit indices");
	*nbfaces_out = nf;
	*nbf_out = nbf;
	*nbq_out = (int)nq;
	if (!face2elem || !fnode2enode || !elem2qnode || !node || (nbf > 0 && !boundaryface))
		return GDN_CUDA_OK; // size query

	int *e2q, *f2e, *fn, *bfd;
	double *nod;
	GDN_CUDA_TRY(B.get(&e2q, 10 * ne + 6LL * nbf));
	GDN_CUDA_TRY(B.get(&f2e, 4LL * nf));
	GDN_CUDA_TRY(B.get(&fn, 12LL * nf));
	GDN_CUDA_TRY(B.get(&bfd, nbf));
	GDN_CUDA_TRY(B.get(&nod, 3 * nq));
	mb_vertex_e2q<<<gf, 256, 0, s>>>(e2n, vmap, ne, e2q);
	GDN_CUDA_TRY(cudaGetLastError());
	mb_vertex_nodes<<<gv, 256, 0, s>>>(used, vmap, nbnodes, crd, nod);
	GDN_CUDA_TRY(cudaGetLastError());
	mb_edge_nodes<<<ge, 256, 0, s>>>(eks, eidxs, head, run, nek, nvq, crd, e2q, nod);
	GDN_CUDA_TRY(cudaGetLastError());
	mb_faces<<<gf, 256, 0, s>>>(e2e, keep, fpos, bpos, ne, e2q, f2e, fn, bfd, bad);
	GDN_CUDA_TRY(cudaGetLastError());
	GDN_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(elem2qnode, e2q, (10 * ne + 6LL * nbf) * sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(face2elem, f2e, 4LL * nf * sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(fnode2enode, fn, 12LL * nf * sizeof(int), cudaMemcpyDeviceToHost, s));
	if (nbf > 0)
		GDN_CUDA_TRY(cudaMemcpyAsync(boundaryface, bfd, nbf * sizeof(int), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaMemcpyAsync(node, nod, 3 * nq * sizeof(double), cudaMemcpyDeviceToHost, s));
	GDN_CUDA_TRY(cudaStreamSynchronize(s));
	if (hbad)
		return gdn_set_error(GDN_CUDA_ERR_MESH, "mesh_build_gpu: face nodes do not match");
	return GDN_CUDA_OK;
}
