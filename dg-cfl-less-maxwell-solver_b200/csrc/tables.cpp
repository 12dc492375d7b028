// P2 (T10) reference-element tables computed from the P2 Lagrange basis.
//
// The node numbering, face numbering and face-node order are the reference's
// (src/mesh/t10.h:26-60, t10.c:23-42): vertices 0..3 at (0,0,0), (1,0,0),
// (0,1,0), (0,0,1); edge nodes 4:(0,1) 5:(1,2) 6:(0,2) 7:(0,3) 8:(1,3) 9:(2,3);
// T4 faces F0 = (0,3,2), F1 = (0,1,3), F2 = (0,2,1), F3 = (1,2,3), each listed
// as (a, b, c, mid(a,b), mid(b,c), mid(c,a)).  These must be alike for the
// state layout and the face permutations to mean the same thing.
//
// Every table entry is an exact rational: the integral of a monomial over the
// unit tetrahedron is a! b! c! / (a+b+c+3)!, and over the unit triangle
// a! b! / (a+b+2)!.  Products of P2 basis functions have integer coefficients,
// so sums are carried exactly in 64-bit integers scaled by 7! (tet) or 6!
// (triangle) and divided once, giving correctly rounded doubles.
//
// The face mass is then rounded to 10 significant digits, because the
// reference's t10_face_scal holds 10-digit literals (t10.c:1317-1330) and the
// FP64 path has to reproduce the reference's operator to 1e-12.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/gdon3d_cuda.h"

namespace {

// polynomial in (x, y, z) of total degree <= 4, integer coefficients
struct Poly {
	long long c[5][5][5];
	Poly() { std::memset(c, 0, sizeof(c)); }
};

Poly mul(const Poly &a, const Poly &b)
{
	Poly r;
	for (int i = 0; i < 5; i++)
		for (int j = 0; j < 5; j++)
			for (int k = 0; k < 5; k++) {
				if (!a.c[i][j][k])
					continue;
				for (int p = 0; p + i < 5; p++)
					for (int q = 0; q + j < 5; q++)
						for (int s = 0; s + k < 5; s++)
							if (b.c[p][q][s])
								r.c[i + p][j + q][k + s] += a.c[i][j][k] * b.c[p][q][s];
			}
	return r;
}

Poly add(const Poly &a, const Poly &b, long long sa = 1, long long sb = 1)
{
	Poly r;
	for (int i = 0; i < 5; i++)
		for (int j = 0; j < 5; j++)
			for (int k = 0; k < 5; k++)
				r.c[i][j][k] = sa * a.c[i][j][k] + sb * b.c[i][j][k];
	return r;
}

Poly deriv(const Poly &a, int dir)
{
	Poly r;
	for (int i = 0; i < 5; i++)
		for (int j = 0; j < 5; j++)
			for (int k = 0; k < 5; k++) {
				int e[3] = {i, j, k};
				if (e[dir] == 0)
					continue;
				long long v = a.c[i][j][k] * e[dir];
				e[dir]--;
				r.c[e[0]][e[1]][e[2]] += v;
			}
	return r;
}

long long fact(int n)
{
	long long f = 1;
	for (int i = 2; i <= n; i++)
		f *= i;
	return f;
}

// integral over the unit tetrahedron times 7!
long long int_tet_x5040(const Poly &a)
{
	long long s = 0;
	for (int i = 0; i < 5; i++)
		for (int j = 0; j < 5; j++)
			for (int k = 0; k < 5; k++)
				if (a.c[i][j][k]) {
					int n = i + j + k;
					s += a.c[i][j][k] * fact(i) * fact(j) * fact(k) * (5040 / fact(n + 3));
				}
	return s;
}

// integral over the unit triangle (z ignored, must be 0) times 6!
long long int_tri_x720(const Poly &a)
{
	long long s = 0;
	for (int i = 0; i < 5; i++)
		for (int j = 0; j < 5; j++)
			if (a.c[i][j][0]) {
				int n = i + j;
				s += a.c[i][j][0] * fact(i) * fact(j) * (720 / fact(n + 2));
			}
	return s;
}

Poly mono(long long coef, int i, int j, int k)
{
	Poly p;
	p.c[i][j][k] = coef;
	return p;
}

// barycentric coordinates on the unit tetrahedron
void tet_barycentric(Poly l[4])
{
	l[0] = add(add(mono(1, 0, 0, 0), mono(-1, 1, 0, 0)), add(mono(-1, 0, 1, 0), mono(-1, 0, 0, 1)));
	l[1] = mono(1, 1, 0, 0);
	l[2] = mono(1, 0, 1, 0);
	l[3] = mono(1, 0, 0, 1);
}

const int kEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
const int kT4Face[4][3] = {{0, 3, 2}, {0, 1, 3}, {0, 2, 1}, {1, 2, 3}};

int edge_node(int a, int b)
{
	for (int e = 0; e < 6; e++)
		if ((kEdge[e][0] == a && kEdge[e][1] == b) || (kEdge[e][0] == b && kEdge[e][1] == a))
			return 4 + e;
	return -1;
}

// P2 Lagrange basis: vertex l(2l-1), edge 4 l_a l_b
void p2_basis(const Poly l[], int nvert, const int (*edges)[2], int nedge, Poly *phi)
{
	for (int v = 0; v < nvert; v++)
		phi[v] = add(mul(mono(2, 0, 0, 0), mul(l[v], l[v])), l[v], 1, -1);
	for (int e = 0; e < nedge; e++)
		phi[nvert + e] = mul(mono(4, 0, 0, 0), mul(l[edges[e][0]], l[edges[e][1]]));
}

double round_sig10(double v)
{
	if (v == 0.0)
		return 0.0;
	char buf[64];
	std::snprintf(buf, sizeof(buf), "%.9e", v);
	return std::strtod(buf, nullptr);
}

} // namespace

extern "C" int gdn_cuda_t10_tables(gdn_cuda_tables *t)
{
	if (!t)
		return GDN_CUDA_ERR_INVALID;
	std::memset(t, 0, sizeof(*t));
	Poly l[4], phi[10];
	tet_barycentric(l);
	p2_basis(l, 4, kEdge, 6, phi);

	for (int i = 0; i < 10; i++)
		t->wpg[i] = (double)int_tet_x5040(phi[i]) / 5040.0;
	long long mass_num[10][10];
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++) {
			mass_num[i][j] = int_tet_x5040(mul(phi[i], phi[j]));
			t->mass[i][j] = (double)mass_num[i][j] / 5040.0;
		}
	for (int k = 0; k < 3; k++) {
		Poly d[10];
		for (int i = 0; i < 10; i++)
			d[i] = deriv(phi[i], k);
		for (int i = 0; i < 10; i++)
			for (int j = 0; j < 10; j++)
				t->internal[i][j][k] = (double)int_tet_x5040(mul(d[i], phi[j])) / 5040.0;
	}
	// inverse of the mass matrix: Gauss-Jordan with partial pivoting in long
	// double on the exact integer numerators (M = N / 5040, M^-1 = 5040 N^-1)
	long double a[10][20];
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 20; j++)
			a[i][j] = j < 10 ? (long double)mass_num[i][j] : (j - 10 == i ? 1.0L : 0.0L);
	for (int k = 0; k < 10; k++) {
		int p = k;
		for (int r = k + 1; r < 10; r++)
			if (fabsl(a[r][k]) > fabsl(a[p][k]))
				p = r;
		if (p != k)
			for (int c = 0; c < 20; c++) {
				long double tmp = a[k][c];
				a[k][c] = a[p][c];
				a[p][c] = tmp;
			}
		long double inv = 1.0L / a[k][k];
		for (int c = 0; c < 20; c++)
			a[k][c] *= inv;
		for (int r = 0; r < 10; r++)
			if (r != k && a[r][k] != 0.0L) {
				long double f = a[r][k];
				for (int c = 0; c < 20; c++)
					a[r][c] -= f * a[k][c];
			}
	}
	for (int i = 0; i < 10; i++)
		for (int j = 0; j < 10; j++)
			t->inv_mass[i][j] = (double)(a[i][10 + j] * 5040.0L);

	// P2 triangle mass on the unit triangle (area 1/2), node order
	// (v0, v1, v2, mid01, mid12, mid20)
	Poly lt[3], pt[6];
	lt[0] = add(mono(1, 0, 0, 0), add(mono(-1, 1, 0, 0), mono(-1, 0, 1, 0)));
	lt[1] = mono(1, 1, 0, 0);
	lt[2] = mono(1, 0, 1, 0);
	const int tri_edges[3][2] = {{0, 1}, {1, 2}, {2, 0}};
	p2_basis(lt, 3, tri_edges, 3, pt);
	for (int i = 0; i < 6; i++)
		for (int j = 0; j < 6; j++)
			t->face_scal[i][j] = round_sig10((double)int_tri_x720(mul(pt[i], pt[j])) / 720.0);

	const double inv_sqrt3 = (double)(1.0L / sqrtl(3.0L));
	const double rn[4][3] = {{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {inv_sqrt3, inv_sqrt3, inv_sqrt3}};
	for (int f = 0; f < 4; f++) {
		for (int k = 0; k < 3; k++)
			t->ref_normal[f][k] = rn[f][k];
		const int *v = kT4Face[f];
		t->face2node[f][0] = v[0];
		t->face2node[f][1] = v[1];
		t->face2node[f][2] = v[2];
		t->face2node[f][3] = edge_node(v[0], v[1]);
		t->face2node[f][4] = edge_node(v[1], v[2]);
		t->face2node[f][5] = edge_node(v[2], v[0]);
	}
	return GDN_CUDA_OK;
}
