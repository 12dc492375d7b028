/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker.
 *
 * CPU restatement (FP64, matrix-free) of Gdon3d's two hot paths, written from
 * the reference's algorithm; pinned against the reference's own code
 * (oracle/_ref) by tests/test_oracle.py.
 *
 *   RK3      src/dg/explicit.c:39-117 (time loop), src/dg/dg.c:61-107
 *            (boundary update), src/simulation/simulation.c:218-261 (inverse
 *            mass), :263-324 (volume term), :356-491 (face flux),
 *            src/models/maxwell.c:152-192 (upwind flux).
 *   kinetic  src/dg/relaxation.c:24-185 (theta scheme), simulation.c:493-604
 *            (kinetic face flux), src/dg/dg.c:109-147 (relaxation),
 *            src/models/d3q4.c:82-301, src/models/d3q6.c (moment maps).
 *
 * Inputs are the reference's mesh arrays (gdn_mesh after
 * mesh_build_connectivity) and P2 tables; the state uses the reference's wn
 * layout.  Unlike the GPU path this code keeps the reference's structure:
 * each face flux is evaluated once with the L-side normal and added with
 * + to L and - to R; the CFL-less step applies M2 and then solves M1 by a
 * block forward substitution in a topological (downwind) element order with
 * a partial-pivoting LU of each 10x10 diagonal block.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct orc_mesh {
	int nbelems, nbfaces, nboundaryfaces, nbqnodes;
	const int *face2elem, *fnode2enode, *boundaryface, *elem2qnode;
	const double *node;
} orc_mesh;

typedef struct orc_tables {
	double wpg[10];
	double mass[10][10];
	double inv_mass[10][10];
	double internal[10][10][3];
	double face_scal[6][6];
	double ref_normal[4][3];
	int face2node[4][6];
} orc_tables;

typedef struct orc_data {
	int kind;
	double khat[3], kmag, pol[3], amp, phase;
} orc_data;

/* ------------------------------------------------------------ data ---- */
static void exact_w(const orc_data *d, const double *x, double t, double *w)
{
	if (d->kind == 1) { /* maxwell_imposed_macro_cavity, maxwell.c:118-133 */
		const double pi = 0.3141592654e1;
		w[0] = 0;
		w[1] = 0;
		w[2] = sin(pi * x[0]) * sin(pi * x[1]) * cos(sqrt(0.2e1) * pi * t);
		w[3] = -sin(sqrt(0.2e1) * pi * t) * sqrt(0.2e1) * sin(pi * x[0]) * cos(pi * x[1]) / 0.2e1;
		w[4] = sin(sqrt(0.2e1) * pi * t) * sqrt(0.2e1) * cos(pi * x[0]) * sin(pi * x[1]) / 0.2e1;
		w[5] = 0;
		return;
	}
	const double *k = d->khat, *p = d->pol;
	double s = d->amp * sin(d->kmag * ((k[0] * x[0] + k[1] * x[1] + k[2] * x[2]) - t) + d->phase);
	w[0] = p[0] * s;
	w[1] = p[1] * s;
	w[2] = p[2] * s;
	w[3] = (k[1] * p[2] - k[2] * p[1]) * s;
	w[4] = (k[2] * p[0] - k[0] * p[2]) * s;
	w[5] = (k[0] * p[1] - k[1] * p[0]) * s;
}

/* maxwell_num_flux_upwind, maxwell.c:152-192 (same formula). */
static void upwind(const double *wL, const double *wR, const double *n, double *flux)
{
	const double nx = n[0], ny = n[1], nz = n[2];
	const double r = 1.0 / (sqrt(nx * nx + ny * ny + nz * nz) + 1e-16);
	const double nxy = r * nx * ny, nxz = r * nx * nz, nyz = r * ny * nz;
	const double nxx = r * nx * nx, nyy = r * ny * ny, nzz = r * nz * nz;
	double Es[3], Hs[3], Ed[3], Hd[3];
	for (int c = 0; c < 3; c++) {
		Es[c] = 0.5 * (wR[c] + wL[c]);
		Hs[c] = 0.5 * (wR[3 + c] + wL[3 + c]);
		Ed[c] = 0.5 * (wR[c] - wL[c]);
		Hd[c] = 0.5 * (wR[3 + c] - wL[3 + c]);
	}
	flux[0] = nz * Hs[1] - ny * Hs[2] - (nyy + nzz) * Ed[0] + nxy * Ed[1] + nxz * Ed[2];
	flux[1] = -nz * Hs[0] + nx * Hs[2] + nxy * Ed[0] - (nxx + nzz) * Ed[1] + nyz * Ed[2];
	flux[2] = -nx * Hs[1] + ny * Hs[0] + nxz * Ed[0] + nyz * Ed[1] - (nxx + nyy) * Ed[2];
	flux[3] = -nz * Es[1] + ny * Es[2] - (nyy + nzz) * Hd[0] + nxy * Hd[1] + nxz * Hd[2];
	flux[4] = nz * Es[0] - nx * Es[2] + nxy * Hd[0] - (nxx + nzz) * Hd[1] + nyz * Hd[2];
	flux[5] = -ny * Es[0] + nx * Es[1] + nxz * Hd[0] + nyz * Hd[1] - (nxx + nyy) * Hd[2];
}

/* ------------------------------------------------------- geometry ---- */
static void elem_geometry(const orc_mesh *m, int e, double cod[3][3], double *det)
{
	double p[4][3], dt[3][3];
	for (int v = 0; v < 4; v++)
		for (int c = 0; c < 3; c++)
			p[v][c] = m->node[3 * m->elem2qnode[10 * e + v] + c];
	for (int i = 0; i < 3; i++)
		for (int j = 0; j < 3; j++)
			dt[i][j] = p[j + 1][i] - p[0][i];
	cod[0][0] = dt[1][1] * dt[2][2] - dt[1][2] * dt[2][1];
	cod[0][1] = -dt[1][0] * dt[2][2] + dt[1][2] * dt[2][0];
	cod[0][2] = dt[1][0] * dt[2][1] - dt[1][1] * dt[2][0];
	cod[1][0] = -dt[0][1] * dt[2][2] + dt[0][2] * dt[2][1];
	cod[1][1] = dt[0][0] * dt[2][2] - dt[0][2] * dt[2][0];
	cod[1][2] = -dt[0][0] * dt[2][1] + dt[0][1] * dt[2][0];
	cod[2][0] = dt[0][1] * dt[1][2] - dt[0][2] * dt[1][1];
	cod[2][1] = -dt[0][0] * dt[1][2] + dt[0][2] * dt[1][0];
	cod[2][2] = dt[0][0] * dt[1][1] - dt[0][1] * dt[1][0];
	*det = dt[0][0] * cod[0][0] + dt[0][1] * cod[0][1] + dt[0][2] * cod[0][2];
}

/* L-side scaled normal of face F (simulation.c:369-395) */
static void face_normal(const orc_mesh *m, const orc_tables *t, int F, double vn[3])
{
	double cod[3][3], det;
	const int eL = m->face2elem[4 * F], fL = m->face2elem[4 * F + 1];
	elem_geometry(m, eL, cod, &det);
	for (int i = 0; i < 3; i++) {
		vn[i] = 0.0;
		for (int j = 0; j < 3; j++)
			vn[i] += cod[i][j] * t->ref_normal[fL][j];
	}
	if (fL == 3)
		for (int i = 0; i < 3; i++)
			vn[i] *= sqrt(3);
}

/* per element and local face: face id and side (0 = L, 1 = R) */
typedef struct {
	int *face, *side, *bidx;
	double *det, *cod, *vn;
} orc_topo;

static void topo_build(const orc_mesh *m, const orc_tables *t, orc_topo *tp)
{
	const int ne = m->nbelems, nf = m->nbfaces;
	tp->face = (int *)malloc(sizeof(int) * 4 * ne);
	tp->side = (int *)malloc(sizeof(int) * 4 * ne);
	tp->bidx = (int *)malloc(sizeof(int) * nf);
	tp->det = (double *)malloc(sizeof(double) * ne);
	tp->cod = (double *)malloc(sizeof(double) * 9 * ne);
	tp->vn = (double *)malloc(sizeof(double) * 3 * nf);
	for (int F = 0; F < nf; F++) {
		tp->bidx[F] = -1;
		const int eL = m->face2elem[4 * F], fL = m->face2elem[4 * F + 1];
		const int eR = m->face2elem[4 * F + 2], fR = m->face2elem[4 * F + 3];
		tp->face[4 * eL + fL] = F;
		tp->side[4 * eL + fL] = 0;
		if (eR >= 0) {
			tp->face[4 * eR + fR] = F;
			tp->side[4 * eR + fR] = 1;
		}
		face_normal(m, t, F, tp->vn + 3 * F);
	}
	for (int b = 0; b < m->nboundaryfaces; b++)
		tp->bidx[m->boundaryface[b]] = b;
	for (int e = 0; e < ne; e++) {
		double cod[3][3];
		elem_geometry(m, e, cod, tp->det + e);
		memcpy(tp->cod + 9 * e, cod, sizeof(cod));
	}
}

static void topo_free(orc_topo *tp)
{
	free(tp->face);
	free(tp->side);
	free(tp->bidx);
	free(tp->det);
	free(tp->cod);
	free(tp->vn);
}

/* ---------------------------------------------------------- HP-1 ---- */
/* F w restricted to the volume dofs of element e (RK3), reference layout
 * wn[ipg * 6 + iw]. */
static void rk3_residual_elem(const orc_mesh *m, const orc_tables *t, const orc_topo *tp, const double *w,
							  int e, double R[10][6])
{
	const int ne = m->nbelems, off = 10 * ne;
	const double *cod = tp->cod + 9 * e;
	memset(R, 0, sizeof(double) * 60);
	/* volume: row (ii, k) col (jj, l) = -[A(c_ij) e_k]_l, simulation.c:263-324 */
	for (int ii = 0; ii < 10; ii++)
		for (int jj = 0; jj < 10; jj++) {
			double cg[3] = {0, 0, 0};
			for (int l = 0; l < 3; l++)
				for (int k = 0; k < 3; k++)
					cg[l] += cod[3 * l + k] * t->internal[ii][jj][k];
			const double *wj = w + 6 * (10 * e + jj);
			double fl[6];
			upwind(wj, wj, cg, fl); /* = A(c) wj, A symmetric */
			for (int k = 0; k < 6; k++)
				R[ii][k] -= fl[k];
		}
	/* faces: Phi_ii = sum_jj S[ii][jj] F(wL_jj, wR_jj, vn_L); L += Phi, R -= Phi */
	for (int lf = 0; lf < 4; lf++) {
		const int F = tp->face[4 * e + lf], side = tp->side[4 * e + lf];
		const int eL = m->face2elem[4 * F], eR = m->face2elem[4 * F + 2];
		const int *fn = m->fnode2enode + 12 * F;
		double flux[6][6];
		for (int jj = 0; jj < 6; jj++) {
			const double *wL = w + 6 * (10 * eL + fn[jj]);
			const double *wR = eR >= 0 ? w + 6 * (10 * eR + fn[6 + jj])
									   : w + 6 * (off + 6 * tp->bidx[F] + fn[6 + jj]);
			upwind(wL, wR, tp->vn + 3 * F, flux[jj]);
		}
		for (int ii = 0; ii < 6; ii++) {
			const int node = side == 0 ? fn[ii] : fn[6 + ii];
			const double sg = side == 0 ? 1.0 : -1.0;
			for (int jj = 0; jj < 6; jj++)
				for (int k = 0; k < 6; k++)
					R[node][k] += sg * t->face_scal[ii][jj] * flux[jj][k];
		}
	}
}

static void boundary_rk3(const orc_mesh *m, const orc_tables *t, const orc_data *d, double tt, double *w)
{
	const int off = 10 * m->nbelems;
	for (int b = 0; b < m->nboundaryfaces; b++) {
		const int F = m->boundaryface[b], eL = m->face2elem[4 * F];
		for (int j = 0; j < 6; j++) {
			const double *x = m->node + 3 * m->elem2qnode[10 * eL + m->fnode2enode[12 * F + j]];
			exact_w(d, x, tt, w + 6 * (off + 6 * b + j));
		}
	}
	(void)t;
}

/* dg_solve_rk3 (explicit.c:39-117) on the reference wn layout. */
int orc_rk3_run(const orc_mesh *m, const orc_tables *t, const orc_data *d, double dt, int steps, double *wn,
				double *t_out)
{
	const double A[3] = {0., -5. / 9., -153. / 128.};
	const double B[3] = {1. / 3., 15. / 16., 8. / 15.};
	const double Cc[3] = {0., 1. / 3., 3. / 4.};
	const int ne = m->nbelems;
	const long long size = 6LL * (10LL * ne + 6LL * m->nboundaryfaces);
	orc_topo tp;
	topo_build(m, t, &tp);
	double *k2 = (double *)calloc(size, sizeof(double));
	double *dw = (double *)calloc(size, sizeof(double));
	memset(wn, 0, sizeof(double) * size);
	for (int e = 0; e < ne; e++) /* dg_init_sol_macro, dg.c:32-59 */
		for (int i = 0; i < 10; i++)
			exact_w(d, m->node + 3 * m->elem2qnode[10 * e + i], 0.0, wn + 6 * (10 * e + i));
	double tt = 0.0;
	for (int it = 0; it < steps; it++) {
		for (int s = 0; s < 3; s++) {
			boundary_rk3(m, t, d, tt + Cc[s] * dt, wn);
#pragma omp parallel for schedule(static)
			for (int e = 0; e < ne; e++) {
				double R[10][6];
				rk3_residual_elem(m, t, &tp, wn, e, R);
				for (int i = 0; i < 10; i++)
					for (int k = 0; k < 6; k++) {
						double acc = 0.0;
						for (int j = 0; j < 10; j++)
							acc += t->inv_mass[i][j] / tp.det[e] * R[j][k];
						dw[6 * (10 * e + i) + k] = acc;
					}
			}
			/* boundary dofs: identity mass, zero flux -> dw = 0 */
#pragma omp parallel for schedule(static)
			for (long long j = 0; j < size; j++) {
				k2[j] = (s == 0 ? 0.0 : A[s] * k2[j]) - dt * dw[j];
				wn[j] = wn[j] + B[s] * k2[j];
			}
		}
		tt += dt;
	}
	*t_out = tt;
	free(k2);
	free(dw);
	topo_free(&tp);
	return 0;
}

/* simulation_error_l2 (simulation.c:606-666); scheme 0 RK3, else kinetic
 * with nb_v velocities. */
double orc_error_l2(const orc_mesh *m, const orc_tables *t, const orc_data *d, int nb_v, const double *wn,
					double tt)
{
	const int ne = m->nbelems;
	const long long neq = 10LL * ne + 6LL * m->nboundaryfaces;
	double err[6] = {0, 0, 0, 0, 0, 0};
	for (int e = 0; e < ne; e++) {
		double cod[3][3], det;
		elem_geometry(m, e, cod, &det);
		for (int i = 0; i < 10; i++) {
			const long long ipg = 10LL * e + i;
			double wex[6], wl[6];
			exact_w(d, m->node + 3 * m->elem2qnode[ipg], tt, wex);
			for (int k = 0; k < 6; k++) {
				if (nb_v == 0) {
					wl[k] = wn[6 * ipg + k];
				} else {
					wl[k] = 0.0;
					for (int v = 0; v < nb_v; v++)
						wl[k] += wn[(long long)(k * nb_v + v) * neq + ipg];
				}
				const double diff = wl[k] - wex[k];
				err[k] += diff * diff * t->wpg[i] * det;
			}
		}
	}
	double e2 = 0.0;
	for (int k = 0; k < 6; k++)
		e2 += sqrt(fabs(err[k])) / 6;
	return e2;
}

/* ---------------------------------------------------------- HP-2 ---- */
typedef struct {
	int nb_v;
	double vi[18];
	double lambda, omega, theta;
} orc_kin;

/* f_eq(w) for d3q4 (d3q4.c:137-191, 261-273) and d3q6 (d3q6.c:154-219,
 * 319-331): q_d = A(e_d) w from the flux with wL = wR = w. */
static void feq(const orc_kin *km, const double *w, double *f /* [iw*nb_v + iv] */)
{
	double q[3][6];
	const double e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
	for (int dd = 0; dd < 3; dd++)
		upwind(w, w, e[dd], q[dd]);
	const double l = km->lambda, l2 = l * l;
	for (int iw = 0; iw < 6; iw++)
		for (int iv = 0; iv < km->nb_v; iv++) {
			const double *v = km->vi + 3 * iv;
			if (km->nb_v == 4) {
				f[iw * 4 + iv] = (w[iw] + (q[0][iw] * v[0] + q[1][iw] * v[1] + q[2][iw] * v[2]) / l2) / 4;
			} else {
				/* axis velocity: +-lambda e_a */
				const int a = iv % 3;
				const double sg = iv < 3 ? 1.0 : -1.0;
				f[iw * 6 + iv] = w[iw] / 6. + sg * q[a][iw] / (2. * l);
			}
		}
}

static void kin_get(const double *wn, long long neq, int m, long long ipg, double *f)
{
	for (int im = 0; im < m; im++)
		f[im] = wn[im * neq + ipg];
}

static void kin_set(double *wn, long long neq, int m, long long ipg, const double *f)
{
	for (int im = 0; im < m; im++)
		wn[im * neq + ipg] = f[im];
}

static void kin_boundary(const orc_mesh *m, const orc_kin *km, const orc_data *d, double tt, double *wn)
{
	const long long ne = m->nbelems, neq = 10 * ne + 6LL * m->nboundaryfaces;
	const int mm = 6 * km->nb_v;
	for (int b = 0; b < m->nboundaryfaces; b++) {
		const int F = m->boundaryface[b], eL = m->face2elem[4 * F];
		for (int j = 0; j < 6; j++) {
			double wI[6], f[36];
			exact_w(d, m->node + 3 * m->elem2qnode[10 * eL + m->fnode2enode[12 * F + j]], tt, wI);
			feq(km, wI, f);
			kin_set(wn, neq, mm, 10 * ne + 6LL * b + j, f);
		}
	}
}

/* (F_v x) on the volume rows of element e for one scalar component stored
 * at x[ipg] (kinetic matrices, simulation.c:298-308 and 493-604). */
static void kin_F_elem(const orc_mesh *m, const orc_tables *t, const orc_topo *tp, const double *v, const double *x,
					   int e, double out[10])
{
	const long long off = 10LL * m->nbelems;
	const double *cod = tp->cod + 9 * e;
	for (int ii = 0; ii < 10; ii++) {
		double acc = 0.0;
		for (int jj = 0; jj < 10; jj++) {
			double cg[3] = {0, 0, 0};
			for (int l = 0; l < 3; l++)
				for (int k = 0; k < 3; k++)
					cg[l] += cod[3 * l + k] * t->internal[ii][jj][k];
			acc -= (v[0] * cg[0] + v[1] * cg[1] + v[2] * cg[2]) * x[10LL * e + jj];
		}
		out[ii] = acc;
	}
	for (int lf = 0; lf < 4; lf++) {
		const int F = tp->face[4 * e + lf], side = tp->side[4 * e + lf];
		const int eL = m->face2elem[4 * F], eR = m->face2elem[4 * F + 2];
		const int *fn = m->fnode2enode + 12 * F;
		const double *vn = tp->vn + 3 * F;
		const double s = v[0] * vn[0] + v[1] * vn[1] + v[2] * vn[2];
		const double sp = s > 0 ? s : 0, sm = s - sp;
		double g[6];
		for (int jj = 0; jj < 6; jj++) {
			const double xL = x[10LL * eL + fn[jj]];
			const double xR = eR >= 0 ? x[10LL * eR + fn[6 + jj]] : x[off + 6LL * tp->bidx[F] + fn[6 + jj]];
			g[jj] = sp * xL + sm * xR;
		}
		for (int ii = 0; ii < 6; ii++) {
			const int node = side == 0 ? fn[ii] : fn[6 + ii];
			double acc = 0.0;
			for (int jj = 0; jj < 6; jj++)
				acc += t->face_scal[ii][jj] * g[jj];
			out[node] += side == 0 ? acc : -acc;
		}
	}
}

/* The element's own 10x10 block of F_v: the volume term and, on every face,
 * the coupling of the element's rows to its own face values (vnp on the L
 * side, -vnm on the R side). */
static void kin_F_diag(const orc_mesh *m, const orc_tables *t, const orc_topo *tp, const double *v, int e,
					   double Fd[10][10])
{
	const double *cod = tp->cod + 9 * e;
	for (int ii = 0; ii < 10; ii++)
		for (int jj = 0; jj < 10; jj++) {
			double cg[3] = {0, 0, 0};
			for (int l = 0; l < 3; l++)
				for (int k = 0; k < 3; k++)
					cg[l] += cod[3 * l + k] * t->internal[ii][jj][k];
			Fd[ii][jj] = -(v[0] * cg[0] + v[1] * cg[1] + v[2] * cg[2]);
		}
	for (int lf = 0; lf < 4; lf++) {
		const int F = tp->face[4 * e + lf], side = tp->side[4 * e + lf];
		const int *fn = m->fnode2enode + 12 * F;
		const double *vn = tp->vn + 3 * F;
		const double s = v[0] * vn[0] + v[1] * vn[1] + v[2] * vn[2];
		const double sp = s > 0 ? s : 0, sm = s - sp;
		for (int ii = 0; ii < 6; ii++)
			for (int jj = 0; jj < 6; jj++) {
				if (side == 0)
					Fd[fn[ii]][fn[jj]] += t->face_scal[ii][jj] * sp;
				else
					Fd[fn[6 + ii]][fn[6 + jj]] -= t->face_scal[ii][jj] * sm;
			}
	}
}

/* dense LU with partial pivoting, in place; returns 0 on success */
static int lu10(double a[10][10], int piv[10])
{
	for (int k = 0; k < 10; k++) {
		int p = k;
		for (int r = k + 1; r < 10; r++)
			if (fabs(a[r][k]) > fabs(a[p][k]))
				p = r;
		piv[k] = p;
		if (p != k)
			for (int c = 0; c < 10; c++) {
				double tmp = a[k][c];
				a[k][c] = a[p][c];
				a[p][c] = tmp;
			}
		if (a[k][k] == 0.0)
			return -1;
		for (int r = k + 1; r < 10; r++) {
			a[r][k] /= a[k][k];
			for (int c = k + 1; c < 10; c++)
				a[r][c] -= a[r][k] * a[k][c];
		}
	}
	return 0;
}

static void lu10_solve(double a[10][10], const int piv[10], double b[10])
{
	for (int k = 0; k < 10; k++)
		if (piv[k] != k) {
			double tmp = b[k];
			b[k] = b[piv[k]];
			b[piv[k]] = tmp;
		}
	for (int r = 1; r < 10; r++)
		for (int c = 0; c < r; c++)
			b[r] -= a[r][c] * b[c];
	for (int r = 9; r >= 0; r--) {
		for (int c = r + 1; c < 10; c++)
			b[r] -= a[r][c] * b[c];
		b[r] /= a[r][r];
	}
}

/* dg_solve_relaxation (relaxation.c:129-185) on the reference wn layout. */
int orc_kin_run(const orc_mesh *m, const orc_tables *t, const orc_data *d, const orc_kin *km, double dt, int steps,
				double *wn, double *t_out)
{
	const int ne = m->nbelems, nv = km->nb_v, mm = 6 * nv;
	const long long neq = 10LL * ne + 6LL * m->nboundaryfaces;
	const double th = km->theta;
	orc_topo tp;
	topo_build(m, t, &tp);
	memset(wn, 0, sizeof(double) * mm * neq);
	for (int e = 0; e < ne; e++) /* dg_init_sol_macro, kinetic branch */
		for (int i = 0; i < 10; i++) {
			double wI[6], f[36];
			exact_w(d, m->node + 3 * m->elem2qnode[10 * e + i], 0.0, wI);
			feq(km, wI, f);
			kin_set(wn, neq, mm, 10LL * e + i, f);
		}
	/* per velocity: topological order and LU of the M1 diagonal blocks */
	int *order = (int *)malloc(sizeof(int) * (size_t)ne * nv);
	double *lu = (double *)malloc(sizeof(double) * (size_t)ne * nv * 100);
	int *piv = (int *)malloc(sizeof(int) * (size_t)ne * nv * 10);
	int *indeg = (int *)malloc(sizeof(int) * ne);
	int rc = 0;
	for (int iv = 0; iv < nv && rc == 0; iv++) {
		const double *v = km->vi + 3 * iv;
		int qh = 0, qt = 0;
		int *q = order + (size_t)iv * ne;
		for (int e = 0; e < ne; e++) {
			indeg[e] = 0;
			for (int lf = 0; lf < 4; lf++) {
				const int F = tp.face[4 * e + lf];
				if (m->face2elem[4 * F + 2] < 0)
					continue;
				const double *vn = tp.vn + 3 * F;
				const double s = v[0] * vn[0] + v[1] * vn[1] + v[2] * vn[2];
				if ((tp.side[4 * e + lf] == 0 && s < 0) || (tp.side[4 * e + lf] == 1 && s > 0))
					indeg[e]++;
			}
			if (indeg[e] == 0)
				q[qt++] = e;
		}
		while (qh < qt) {
			const int e = q[qh++];
			for (int lf = 0; lf < 4; lf++) {
				const int F = tp.face[4 * e + lf];
				const int eL = m->face2elem[4 * F], eR = m->face2elem[4 * F + 2];
				if (eR < 0)
					continue;
				const double *vn = tp.vn + 3 * F;
				const double s = v[0] * vn[0] + v[1] * vn[1] + v[2] * vn[2];
				int down = -1;
				if (tp.side[4 * e + lf] == 0 && s > 0)
					down = eR;
				if (tp.side[4 * e + lf] == 1 && s < 0)
					down = eL;
				if (down >= 0 && --indeg[down] == 0)
					q[qt++] = down;
			}
		}
		if (qt != ne) {
			rc = -1;
			break;
		}
		/* diagonal block of M1 = I + theta dt Minv/det F_v for each element */
#pragma omp parallel for schedule(static)
		for (int e = 0; e < ne; e++) {
			double Fd[10][10], blk[10][10];
			kin_F_diag(m, t, &tp, v, e, Fd);
			for (int ii = 0; ii < 10; ii++)
				for (int jj = 0; jj < 10; jj++) {
					double acc = 0.0;
					for (int k = 0; k < 10; k++)
						acc += t->inv_mass[ii][k] / tp.det[e] * Fd[k][jj];
					blk[ii][jj] = (ii == jj ? 1.0 : 0.0) + th * dt * acc;
				}
			int p[10];
			if (lu10(blk, p) != 0)
				rc = -2;
			memcpy(lu + ((size_t)iv * ne + e) * 100, blk, sizeof(blk));
			memcpy(piv + ((size_t)iv * ne + e) * 10, p, sizeof(p));
		}
	}
	free(indeg);
	double *sol = (double *)malloc(sizeof(double) * mm * neq);
	double tt = 0.0;
	for (int it = 0; it < steps && rc == 0; it++) {
		kin_boundary(m, km, d, tt + dt / 2, wn);
#pragma omp parallel for schedule(dynamic, 1)
		for (int im = 0; im < mm; im++) {
			const int iv = im % nv;
			const double *v = km->vi + 3 * iv;
			const double *x = wn + (long long)im * neq;
			double *y = sol + (long long)im * neq;
			/* sol = M2 x; boundary rows identity */
			for (int e = 0; e < ne; e++) {
				double Fx[10];
				kin_F_elem(m, t, &tp, v, x, e, Fx);
				for (int ii = 0; ii < 10; ii++) {
					double acc = 0.0;
					for (int k = 0; k < 10; k++)
						acc += t->inv_mass[ii][k] / tp.det[e] * Fx[k];
					y[10LL * e + ii] = x[10LL * e + ii] - (1 - th) * dt * acc;
				}
			}
			for (long long j = 10LL * ne; j < neq; j++)
				y[j] = x[j];
			/* M1 y_new = y: block forward substitution in downwind order */
			const int *q = order + (size_t)iv * ne;
			for (int k = 0; k < ne; k++) {
				const int e = q[k];
				double rhs[10], Fo[10];
				/* off-diagonal part: F_v applied to the current y with the
				 * element's own block zeroed */
				double own[10];
				for (int jj = 0; jj < 10; jj++) {
					own[jj] = y[10LL * e + jj];
					y[10LL * e + jj] = 0.0;
				}
				kin_F_elem(m, t, &tp, v, y, e, Fo);
				for (int ii = 0; ii < 10; ii++) {
					double acc = 0.0;
					for (int kk = 0; kk < 10; kk++)
						acc += t->inv_mass[ii][kk] / tp.det[e] * Fo[kk];
					rhs[ii] = own[ii] - th * dt * acc;
				}
				lu10_solve((double(*)[10])(lu + ((size_t)iv * ne + e) * 100), piv + ((size_t)iv * ne + e) * 10,
						   rhs);
				for (int ii = 0; ii < 10; ii++)
					y[10LL * e + ii] = rhs[ii];
			}
		}
		double *tmp = wn; /* swap, relaxation.c:161-163 */
		memcpy(tmp, sol, sizeof(double) * mm * neq);
		/* dg_apply_relaxation, dg.c:109-147 (volume and boundary dofs) */
#pragma omp parallel for schedule(static)
		for (long long ipg = 0; ipg < neq; ipg++) {
			double f[36], w[6], fe[36];
			kin_get(wn, neq, mm, ipg, f);
			for (int iw = 0; iw < 6; iw++) {
				w[iw] = 0;
				for (int iv = 0; iv < nv; iv++)
					w[iw] += f[iw * nv + iv];
			}
			feq(km, w, fe);
			for (int im = 0; im < mm; im++)
				f[im] = km->omega * fe[im] + (1. - km->omega) * f[im];
			kin_set(wn, neq, mm, ipg, f);
		}
		tt += dt;
	}
	if (rc == 0)
		kin_boundary(m, km, d, tt, wn);
	*t_out = tt;
	free(sol);
	free(order);
	free(lu);
	free(piv);
	topo_free(&tp);
	return rc;
}
