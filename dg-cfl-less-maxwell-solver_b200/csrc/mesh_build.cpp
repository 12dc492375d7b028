// Host-side connectivity for callers that do not link the reference: the same
// arrays, with the same conventions, as the reference's
// mesh_build_connectivity (src/mesh/mesh.c:1234-1268):
//   - elem2elem from matching sorted T4 face vertex triples (build_face /
//     build_elem2elem, mesh.c:803-862);
//   - face2elem by looping elements ie and local faces ifa and keeping a face
//     when its neighbour index is < ie, so L is the larger element index and
//     a boundary face has eR = locfaceR = -1 (build_face2elem, mesh.c:971-1016);
//   - boundaryface = boundary faces in face order (mesh.c:875-901);
//   - fnode2enode: L ids are the face's P2 nodes, R ids the matching local
//     nodes of eR, or 0..5 on a boundary face; elem2qnode is extended with the
//     L node of each boundary dof (build_fnode2enode, mesh.c:1122-1175).
// These conventions must be alike: they fix the order of the boundary dofs in
// the state vector and which side of each face the reference's assembly
// calls L.  P2 node ids are our own (vertices, then edges in first-seen
// order); only the coordinates attached to (element, local node) matter.
// Edge-node coordinates are 0.5 a + 0.5 b, bit-identical to the reference's
// gdn_tetra_ref2phy evaluation at the reference edge midpoints.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/gdon3d_cuda.h"
#include "internal.h"

namespace {
const int kT4Face[4][3] = {{0, 3, 2}, {0, 1, 3}, {0, 2, 1}, {1, 2, 3}};
const int kEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
// P2 local nodes of each local face: (a, b, c, mid ab, mid bc, mid ca)
const int kFace2Node[4][6] = {{0, 3, 2, 7, 9, 6}, {0, 1, 3, 4, 8, 7}, {0, 2, 1, 6, 5, 4}, {1, 2, 3, 5, 9, 8}};

struct FaceKey {
	int v[3];
	int elem, loc;
};
} // namespace

extern "C" int gdn_cuda_mesh_build(int nbnodes, const double *coords, int nbelems, const int *elem2node,
								   int *nbfaces_out, int *nbf_out, int *nbq_out, int *face2elem,
								   int *fnode2enode, int *boundaryface, int *elem2qnode, double *node)
{
	if (nbnodes <= 0 || nbelems <= 0 || !coords || !elem2node || !nbfaces_out || !nbf_out || !nbq_out)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "mesh_build: bad arguments");
	const long long ne = nbelems;
	for (long long i = 0; i < 4 * ne; i++)
		if (elem2node[i] < 0 || elem2node[i] >= nbnodes)
			return gdn_set_error(GDN_CUDA_ERR_MESH, "mesh_build: elem2node index out of range");

	// faces and neighbours
	std::vector<FaceKey> faces(4 * ne);
	for (long long ie = 0; ie < ne; ie++)
		for (int f = 0; f < 4; f++) {
			FaceKey &k = faces[4 * ie + f];
			for (int a = 0; a < 3; a++)
				k.v[a] = elem2node[4 * ie + kT4Face[f][a]];
			std::sort(k.v, k.v + 3);
			k.elem = (int)ie;
			k.loc = f;
		}
	std::sort(faces.begin(), faces.end(), [](const FaceKey &a, const FaceKey &b) {
		if (a.v[0] != b.v[0])
			return a.v[0] < b.v[0];
		if (a.v[1] != b.v[1])
			return a.v[1] < b.v[1];
		if (a.v[2] != b.v[2])
			return a.v[2] < b.v[2];
		return a.elem < b.elem;
	});
	std::vector<int> e2e(4 * ne, -1);
	for (size_t i = 0; i + 1 < faces.size(); i++) {
		const FaceKey &a = faces[i], &b = faces[i + 1];
		if (a.v[0] == b.v[0] && a.v[1] == b.v[1] && a.v[2] == b.v[2]) {
			if (i + 2 < faces.size()) {
				const FaceKey &c = faces[i + 2];
				if (c.v[0] == a.v[0] && c.v[1] == a.v[1] && c.v[2] == a.v[2])
					return gdn_set_error(GDN_CUDA_ERR_MESH, "mesh_build: non-manifold face");
			}
			e2e[4 * (long long)a.elem + a.loc] = b.elem;
			e2e[4 * (long long)b.elem + b.loc] = a.elem;
			i++;
		}
	}
	faces.clear();
	faces.shrink_to_fit();

	long long nf = 0, nbf = 0;
	for (long long ie = 0; ie < ne; ie++)
		for (int f = 0; f < 4; f++) {
			int ie2 = e2e[4 * ie + f];
			if (ie2 < ie) {
				nf++;
				if (ie2 < 0)
					nbf++;
			}
		}

	// P2 nodes: used vertices first (in vertex order), then edges
	std::vector<int> vmap(nbnodes, -1);
	int nq = 0;
	for (long long i = 0; i < 4 * ne; i++)
		if (vmap[elem2node[i]] < 0)
			vmap[elem2node[i]] = 0;
	for (int v = 0; v < nbnodes; v++)
		if (vmap[v] == 0)
			vmap[v] = nq++;
	// edges keyed by (min vertex, max vertex)
	std::vector<uint64_t> ekeys(6 * ne);
	for (long long ie = 0; ie < ne; ie++)
		for (int e = 0; e < 6; e++) {
			uint64_t a = (uint64_t)elem2node[4 * ie + kEdge[e][0]];
			uint64_t b = (uint64_t)elem2node[4 * ie + kEdge[e][1]];
			if (a > b)
				std::swap(a, b);
			ekeys[6 * ie + e] = (a << 32) | b;
		}
	std::vector<uint64_t> uniq(ekeys);
	std::sort(uniq.begin(), uniq.end());
	uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
	const int nvq = nq;
	nq += (int)uniq.size();

	*nbfaces_out = (int)nf;
	*nbf_out = (int)nbf;
	*nbq_out = nq;
	if (!face2elem || !fnode2enode || !elem2qnode || !node || (nbf > 0 && !boundaryface))
		return GDN_CUDA_OK; // size query

	for (int v = 0; v < nbnodes; v++)
		if (vmap[v] >= 0)
			for (int c = 0; c < 3; c++)
				node[3LL * vmap[v] + c] = coords[3LL * v + c];
	for (size_t k = 0; k < uniq.size(); k++) {
		int a = (int)(uniq[k] >> 32), b = (int)(uniq[k] & 0xffffffffu);
		for (int c = 0; c < 3; c++)
			node[3LL * (nvq + k) + c] = 0.5 * coords[3LL * a + c] + 0.5 * coords[3LL * b + c];
	}
	for (long long ie = 0; ie < ne; ie++) {
		for (int i = 0; i < 4; i++)
			elem2qnode[10 * ie + i] = vmap[elem2node[4 * ie + i]];
		for (int e = 0; e < 6; e++) {
			uint64_t key = ekeys[6 * ie + e];
			size_t pos = std::lower_bound(uniq.begin(), uniq.end(), key) - uniq.begin();
			elem2qnode[10 * ie + 4 + e] = nvq + (int)pos;
		}
	}

	long long fc = 0, bc = 0;
	for (long long ie = 0; ie < ne; ie++)
		for (int f = 0; f < 4; f++) {
			int ie2 = e2e[4 * ie + f];
			if (ie2 >= ie)
				continue;
			face2elem[4 * fc + 0] = (int)ie;
			face2elem[4 * fc + 1] = f;
			face2elem[4 * fc + 2] = ie2;
			face2elem[4 * fc + 3] = -1;
			if (ie2 >= 0) {
				for (int f2 = 0; f2 < 4; f2++)
					if (e2e[4LL * ie2 + f2] == ie) {
						face2elem[4 * fc + 3] = f2;
						break;
					}
			}
			for (int j = 0; j < 6; j++) {
				int inoe = kFace2Node[f][j];
				fnode2enode[12 * fc + j] = inoe;
				int gq = elem2qnode[10 * ie + inoe];
				if (ie2 < 0) {
					fnode2enode[12 * fc + 6 + j] = j;
					elem2qnode[10 * ne + 6 * bc + j] = gq;
				} else {
					int r = 0;
					while (r < 10 && elem2qnode[10LL * ie2 + r] != gq)
						r++;
					if (r == 10)
						return gdn_set_error(GDN_CUDA_ERR_MESH, "mesh_build: face nodes do not match");
					fnode2enode[12 * fc + 6 + j] = r;
				}
			}
			if (ie2 < 0)
				boundaryface[bc++] = (int)fc;
			fc++;
		}
	return GDN_CUDA_OK;
}

// mesh_get_t4_hmin (src/mesh/mesh.c:149-210): min over elements of
// volume / surface, the volume as sum_i w_i det with the T4 weights 1/24 and
// the surface from the scaled face normals.
extern "C" int gdn_cuda_mesh_hmin(const gdn_cuda_mesh *m, double *hmin)
{
	if (!m || !hmin || m->nbelems <= 0 || !m->elem2qnode || !m->node)
		return gdn_set_error(GDN_CUDA_ERR_INVALID, "mesh_hmin: bad arguments");
	double h = 3.4028234663852886e38; // FLT_MAX, as the reference starts from
	const double test[4] = {0.5, 0.5, 0.5, 0.86602540378443865};
	const double rn3 = 0.57735026918962584;
	const double nref[4][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {rn3, rn3, rn3}};
	for (long long ie = 0; ie < m->nbelems; ie++) {
		double p[4][3];
		for (int v = 0; v < 4; v++)
			for (int c = 0; c < 3; c++)
				p[v][c] = m->node[3LL * m->elem2qnode[10 * ie + v] + c];
		double g[3][3], cof[3][3], det;
		gdn_geometry_from_vertices(p, g, cof, &det);
		double vol = 0.0;
		for (int k = 0; k < 4; k++)
			vol += 0.041666666666666667 * det;
		double surf = 0.0;
		for (int f = 0; f < 4; f++) {
			double vn[3];
			for (int a = 0; a < 3; a++) {
				vn[a] = 0.0;
				for (int b = 0; b < 3; b++)
					vn[a] += cof[a][b] * nref[f][b];
			}
			surf += std::sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]) * test[f];
		}
		double loc = vol / surf;
		if (loc < h)
			h = loc;
	}
	*hmin = h;
	return GDN_CUDA_OK;
}
