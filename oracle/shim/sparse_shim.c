/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * Repo-owned implementation of the reference's sparse operator API
 * (prototypes in shim/maths/sparse.h, mirroring src/maths/sparse.h:42-77).
 * The reference backs this API with SuiteSparse CXSparse + KLU (absent here;
 * the reference pins no version of either).  This file is written from the
 * mathematics only:
 *   - COO triplets are appended in insertion order; the CSR form sums
 *     duplicate (i, j) entries in insertion order (the reference's
 *     sparse_csr_allocate, src/maths/sparse.c:176-213, also reduces
 *     duplicates; its CSR is what every later product sees).
 *   - sparse_spmdv: res = A x over CSR rows, OpenMP over rows
 *     (src/maths/sparse.c:387-402).  The accumulator is private per row.
 *   - SpGEMM (src/maths/sparse.c:318-342): Gustavson row-by-row product.
 *   - alpha*A + beta*B (src/maths/sparse.c:361-375).
 *   - Direct solve (replaces klu_analyze/klu_factor/klu_tsolve,
 *     src/maths/sparse.c:411-466): Tarjan's strongly connected components of
 *     the row-dependency graph give a block triangular order; each diagonal
 *     block is factored once by dense LU with partial pivoting; a solve is a
 *     block forward substitution in that order, in place on rhs.  For the
 *     CFL-less transport matrices (block lower triangular in a downwind
 *     element order) this is an exact direct solve like KLU's BTF + LU.
 */
#include <assert.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "maths/sparse.h"

struct gdn_sparse {
	int n;
	/* COO */
	int has_coo;
	long long coo_n, coo_cap;
	int *ci, *cj;
	double *cv;
	/* CSR */
	int has_csr;
	long long *rp;
	int *col;
	double *val;
	/* block triangular LU */
	int has_sym, has_lu;
	int nblk;
	int *blk_ptr; /* nblk + 1 */
	int *blk_idx; /* n: global indices, grouped by block, blocks in solve order */
	int *blk_of; /* n: block id of each index */
	long long *lu_ptr; /* nblk + 1 */
	double *lu; /* dense LU factors, row-major per block */
	int *piv; /* n: local pivot row per block position */
	int max_blk;
};

static void *xmalloc(size_t sz)
{
	void *p = malloc(sz ? sz : 1);
	assert(p);
	return p;
}

gdn_sparse *gdn_sparse_malloc()
{
	gdn_sparse *M = (gdn_sparse *)calloc(1, sizeof(gdn_sparse));
	assert(M);
	return M;
}

gdn_sparse *sparse_coo_init(int n)
{
	gdn_sparse *M = gdn_sparse_malloc();
	M->n = n;
	M->has_coo = 1;
	M->coo_cap = 1024;
	M->ci = (int *)xmalloc(sizeof(int) * M->coo_cap);
	M->cj = (int *)xmalloc(sizeof(int) * M->coo_cap);
	M->cv = (double *)xmalloc(sizeof(double) * M->coo_cap);
	return M;
}

void sparse_coo_insert(gdn_sparse *M, int i, int j, gdn_real val)
{
	assert(M->has_coo);
	assert(i >= 0 && i < M->n && j >= 0 && j < M->n);
	if (M->coo_n == M->coo_cap) {
		M->coo_cap *= 2;
		M->ci = (int *)realloc(M->ci, sizeof(int) * M->coo_cap);
		M->cj = (int *)realloc(M->cj, sizeof(int) * M->coo_cap);
		M->cv = (double *)realloc(M->cv, sizeof(double) * M->coo_cap);
		assert(M->ci && M->cj && M->cv);
	}
	M->ci[M->coo_n] = i;
	M->cj[M->coo_n] = j;
	M->cv[M->coo_n] = val;
	M->coo_n++;
}

void gdn_sparse_coo_switch_on(gdn_sparse *M, int i, int j)
{
	sparse_coo_insert(M, i, j, 0.);
}

gdn_sparse *sparse_coo_init_identity(int n)
{
	gdn_sparse *Id = sparse_coo_init(n);
	for (int i = 0; i < n; i++)
		sparse_coo_insert(Id, i, i, 1.);
	return Id;
}

static void free_coo(gdn_sparse *M)
{
	free(M->ci);
	free(M->cj);
	free(M->cv);
	M->ci = M->cj = NULL;
	M->cv = NULL;
	M->has_coo = 0;
	M->coo_n = M->coo_cap = 0;
}

static void free_csr(gdn_sparse *M)
{
	free(M->rp);
	free(M->col);
	free(M->val);
	M->rp = NULL;
	M->col = NULL;
	M->val = NULL;
	M->has_csr = 0;
}

static void free_lu(gdn_sparse *M)
{
	free(M->blk_ptr);
	free(M->blk_idx);
	free(M->blk_of);
	free(M->lu_ptr);
	free(M->lu);
	free(M->piv);
	M->blk_ptr = M->blk_idx = M->blk_of = M->piv = NULL;
	M->lu_ptr = NULL;
	M->lu = NULL;
	M->has_sym = M->has_lu = 0;
}

void sparse_free(gdn_sparse *M)
{
	if (!M)
		return;
	free_coo(M);
	free_csr(M);
	free_lu(M);
	free(M);
}

/* Sort key for entries of one row: column, then insertion sequence. */
typedef struct {
	int col;
	long long seq;
	double val;
} row_entry;

static int cmp_row_entry(const void *a, const void *b)
{
	const row_entry *x = (const row_entry *)a, *y = (const row_entry *)b;
	if (x->col != y->col)
		return x->col < y->col ? -1 : 1;
	return x->seq < y->seq ? -1 : (x->seq > y->seq);
}

void sparse_csr_allocate(gdn_sparse *M, bool free_coo_flag)
{
	assert(M->has_coo);
	const int n = M->n;
	const long long nz = M->coo_n;
	if (M->has_csr)
		free_csr(M);

	/* stable counting sort of triplets by row */
	long long *cnt = (long long *)calloc(n + 1, sizeof(long long));
	for (long long k = 0; k < nz; k++)
		cnt[M->ci[k] + 1]++;
	for (int i = 0; i < n; i++)
		cnt[i + 1] += cnt[i];
	long long *pos = (long long *)xmalloc(sizeof(long long) * (n + 1));
	memcpy(pos, cnt, sizeof(long long) * (n + 1));
	row_entry *ent = (row_entry *)xmalloc(sizeof(row_entry) * (nz ? nz : 1));
	for (long long k = 0; k < nz; k++) {
		long long p = pos[M->ci[k]]++;
		ent[p].col = M->cj[k];
		ent[p].seq = k;
		ent[p].val = M->cv[k];
	}

	/* per row: order by (column, insertion), sum duplicates in insertion order */
	M->rp = (long long *)xmalloc(sizeof(long long) * (n + 1));
	long long out = 0;
	M->rp[0] = 0;
	for (int i = 0; i < n; i++) {
		long long b = cnt[i], e = cnt[i + 1];
		qsort(ent + b, (size_t)(e - b), sizeof(row_entry), cmp_row_entry);
		for (long long k = b; k < e;) {
			long long k2 = k + 1;
			double s = ent[k].val;
			while (k2 < e && ent[k2].col == ent[k].col)
				s += ent[k2++].val;
			ent[out].col = ent[k].col;
			ent[out].val = s;
			out++;
			k = k2;
		}
		M->rp[i + 1] = out;
	}
	M->col = (int *)xmalloc(sizeof(int) * (out ? out : 1));
	M->val = (double *)xmalloc(sizeof(double) * (out ? out : 1));
	for (long long k = 0; k < out; k++) {
		M->col[k] = ent[k].col;
		M->val[k] = ent[k].val;
	}
	free(ent);
	free(pos);
	free(cnt);
	M->has_csr = 1;
	if (free_coo_flag)
		free_coo(M);
}

static long long find_entry(const gdn_sparse *M, int i, int j)
{
	for (long long k = M->rp[i]; k < M->rp[i + 1]; k++)
		if (M->col[k] == j)
			return k;
	return -1;
}

void sparse_csr_add_entry(gdn_sparse *M, int i, int j, gdn_real val)
{
	assert(M->has_csr);
	long long k = find_entry(M, i, j);
	assert(k >= 0);
	M->val[k] += val;
}

void sparse_csr_set_entry(gdn_sparse *M, int i, int j, gdn_real val)
{
	assert(M->has_csr);
	long long k = find_entry(M, i, j);
	assert(k >= 0);
	M->val[k] = val;
}

gdn_real sparse_csr_get_entry(gdn_sparse *M, int i, int j)
{
	assert(M->has_csr);
	long long k = find_entry(M, i, j);
	return k >= 0 ? M->val[k] : 0.;
}

gdn_sparse *sparse_init_copy(gdn_sparse *M)
{
	gdn_sparse *C = sparse_coo_init(M->n);
	if (M->has_coo)
		for (long long k = 0; k < M->coo_n; k++)
			sparse_coo_insert(C, M->ci[k], M->cj[k], M->cv[k]);
	if (M->has_csr) {
		long long nz = M->rp[M->n];
		C->rp = (long long *)xmalloc(sizeof(long long) * (M->n + 1));
		C->col = (int *)xmalloc(sizeof(int) * (nz ? nz : 1));
		C->val = (double *)xmalloc(sizeof(double) * (nz ? nz : 1));
		memcpy(C->rp, M->rp, sizeof(long long) * (M->n + 1));
		memcpy(C->col, M->col, sizeof(int) * nz);
		memcpy(C->val, M->val, sizeof(double) * nz);
		C->has_csr = 1;
	}
	if (M->has_sym)
		sparse_solver_init(C);
	if (M->has_lu)
		sparse_solver_lu_factor(C);
	return C;
}

/* Row-wise combination used by both SpGEMM and addition: rows are built with a
 * dense accumulator and a marker; columns keep first-appearance order. */
typedef struct {
	double *acc;
	int *mark;
	int *cols;
} row_ws;

gdn_sparse *sparse_csr_matrix_multiplication(const gdn_sparse *A,
                                             const gdn_sparse *B)
{
	assert(A->has_csr && B->has_csr && A->n == B->n);
	const int n = A->n;
	gdn_sparse *C = gdn_sparse_malloc();
	C->n = n;
	long long *rowcnt = (long long *)calloc(n + 1, sizeof(long long));

#pragma omp parallel
	{
		int *mark = (int *)xmalloc(sizeof(int) * n);
		for (int j = 0; j < n; j++)
			mark[j] = -1;
#pragma omp for schedule(static)
		for (int i = 0; i < n; i++) {
			long long c = 0;
			for (long long ka = A->rp[i]; ka < A->rp[i + 1]; ka++) {
				int k = A->col[ka];
				for (long long kb = B->rp[k]; kb < B->rp[k + 1]; kb++) {
					int j = B->col[kb];
					if (mark[j] != i) {
						mark[j] = i;
						c++;
					}
				}
			}
			rowcnt[i + 1] = c;
		}
		free(mark);
	}
	for (int i = 0; i < n; i++)
		rowcnt[i + 1] += rowcnt[i];
	const long long nz = rowcnt[n];
	C->rp = rowcnt;
	C->col = (int *)xmalloc(sizeof(int) * (nz ? nz : 1));
	C->val = (double *)xmalloc(sizeof(double) * (nz ? nz : 1));

#pragma omp parallel
	{
		int *mark = (int *)xmalloc(sizeof(int) * n);
		double *acc = (double *)xmalloc(sizeof(double) * n);
		for (int j = 0; j < n; j++)
			mark[j] = -1;
#pragma omp for schedule(static)
		for (int i = 0; i < n; i++) {
			long long p0 = C->rp[i], p = p0;
			for (long long ka = A->rp[i]; ka < A->rp[i + 1]; ka++) {
				int k = A->col[ka];
				double a = A->val[ka];
				for (long long kb = B->rp[k]; kb < B->rp[k + 1]; kb++) {
					int j = B->col[kb];
					if (mark[j] != i) {
						mark[j] = i;
						acc[j] = a * B->val[kb];
						C->col[p++] = j;
					} else {
						acc[j] += a * B->val[kb];
					}
				}
			}
			for (long long q = p0; q < p; q++)
				C->val[q] = acc[C->col[q]];
		}
		free(mark);
		free(acc);
	}
	C->has_csr = 1;
	return C;
}

gdn_sparse *sparse_csr_matrix_addition(const gdn_sparse *A, const gdn_sparse *B,
                                       const gdn_real alpha,
                                       const gdn_real beta)
{
	assert(A->has_csr && B->has_csr && A->n == B->n);
	const int n = A->n;
	gdn_sparse *C = gdn_sparse_malloc();
	C->n = n;
	long long cap = A->rp[n] + B->rp[n];
	C->rp = (long long *)xmalloc(sizeof(long long) * (n + 1));
	C->col = (int *)xmalloc(sizeof(int) * (cap ? cap : 1));
	C->val = (double *)xmalloc(sizeof(double) * (cap ? cap : 1));
	int *mark = (int *)xmalloc(sizeof(int) * n);
	long long *where = (long long *)xmalloc(sizeof(long long) * n);
	for (int j = 0; j < n; j++)
		mark[j] = -1;
	long long p = 0;
	C->rp[0] = 0;
	for (int i = 0; i < n; i++) {
		for (long long k = A->rp[i]; k < A->rp[i + 1]; k++) {
			int j = A->col[k];
			mark[j] = i;
			where[j] = p;
			C->col[p] = j;
			C->val[p] = alpha * A->val[k];
			p++;
		}
		for (long long k = B->rp[i]; k < B->rp[i + 1]; k++) {
			int j = B->col[k];
			if (mark[j] == i) {
				C->val[where[j]] += beta * B->val[k];
			} else {
				mark[j] = i;
				where[j] = p;
				C->col[p] = j;
				C->val[p] = beta * B->val[k];
				p++;
			}
		}
		C->rp[i + 1] = p;
	}
	free(mark);
	free(where);
	C->has_csr = 1;
	return C;
}

void sparse_spmdv(const gdn_sparse *A, const gdn_real *x, gdn_real *res)
{
	assert(A->has_csr);
	const int n = A->n;
#pragma omp parallel for schedule(static)
	for (int i = 0; i < n; i++) {
		double s = 0.;
		for (long long k = A->rp[i]; k < A->rp[i + 1]; k++)
			s += A->val[k] * x[A->col[k]];
		res[i] = s;
	}
}

/* Tarjan's algorithm, iterative.  Edge i -> j for every stored a_ij with
 * j != i (row i needs x_j).  Components are emitted after every component
 * they reach, which is exactly a valid block forward-substitution order. */
void sparse_solver_init(gdn_sparse *M)
{
	if (!M->has_csr)
		sparse_csr_allocate(M, true);
	if (M->has_sym)
		free_lu(M);
	const int n = M->n;
	int *index = (int *)xmalloc(sizeof(int) * n);
	int *low = (int *)xmalloc(sizeof(int) * n);
	char *onstk = (char *)calloc(n, 1);
	int *stk = (int *)xmalloc(sizeof(int) * n);
	int *cs_node = (int *)xmalloc(sizeof(int) * n);
	long long *cs_edge = (long long *)xmalloc(sizeof(long long) * n);
	M->blk_of = (int *)xmalloc(sizeof(int) * n);
	M->blk_idx = (int *)xmalloc(sizeof(int) * n);
	M->blk_ptr = (int *)xmalloc(sizeof(int) * (n + 1));
	for (int i = 0; i < n; i++)
		index[i] = -1;
	int counter = 0, sp = 0, nblk = 0, nout = 0;
	M->blk_ptr[0] = 0;
	for (int root = 0; root < n; root++) {
		if (index[root] >= 0)
			continue;
		int csp = 0;
		cs_node[csp] = root;
		cs_edge[csp] = M->rp[root];
		csp++;
		index[root] = low[root] = counter++;
		stk[sp++] = root;
		onstk[root] = 1;
		while (csp > 0) {
			int v = cs_node[csp - 1];
			long long e = cs_edge[csp - 1];
			if (e < M->rp[v + 1]) {
				cs_edge[csp - 1] = e + 1;
				int w = M->col[e];
				if (w == v)
					continue;
				if (index[w] < 0) {
					index[w] = low[w] = counter++;
					stk[sp++] = w;
					onstk[w] = 1;
					cs_node[csp] = w;
					cs_edge[csp] = M->rp[w];
					csp++;
				} else if (onstk[w] && index[w] < low[v]) {
					low[v] = index[w];
				}
			} else {
				csp--;
				if (csp > 0) {
					int u = cs_node[csp - 1];
					if (low[v] < low[u])
						low[u] = low[v];
				}
				if (low[v] == index[v]) {
					int w;
					do {
						w = stk[--sp];
						onstk[w] = 0;
						M->blk_of[w] = nblk;
						M->blk_idx[nout++] = w;
					} while (w != v);
					nblk++;
					M->blk_ptr[nblk] = nout;
				}
			}
		}
	}
	assert(nout == n);
	M->nblk = nblk;
	M->max_blk = 0;
	for (int b = 0; b < nblk; b++) {
		int s = M->blk_ptr[b + 1] - M->blk_ptr[b];
		if (s > M->max_blk)
			M->max_blk = s;
	}
	free(index);
	free(low);
	free(onstk);
	free(stk);
	free(cs_node);
	free(cs_edge);
	M->has_sym = 1;
}

void sparse_solver_lu_factor(gdn_sparse *M)
{
	if (!M->has_sym)
		sparse_solver_init(M);
	const int nblk = M->nblk;
	M->lu_ptr = (long long *)xmalloc(sizeof(long long) * (nblk + 1));
	M->lu_ptr[0] = 0;
	for (int b = 0; b < nblk; b++) {
		long long s = M->blk_ptr[b + 1] - M->blk_ptr[b];
		M->lu_ptr[b + 1] = M->lu_ptr[b] + s * s;
	}
	M->lu = (double *)calloc((size_t)M->lu_ptr[nblk] + 1, sizeof(double));
	M->piv = (int *)xmalloc(sizeof(int) * (M->n ? M->n : 1));
	int *loc = (int *)xmalloc(sizeof(int) * (M->n ? M->n : 1));

#pragma omp parallel for schedule(dynamic, 64)
	for (int b = 0; b < nblk; b++) {
		const int b0 = M->blk_ptr[b];
		const int s = M->blk_ptr[b + 1] - b0;
		double *a = M->lu + M->lu_ptr[b];
		for (int r = 0; r < s; r++)
			loc[M->blk_idx[b0 + r]] = r;
		for (int r = 0; r < s; r++) {
			int i = M->blk_idx[b0 + r];
			for (long long k = M->rp[i]; k < M->rp[i + 1]; k++) {
				int j = M->col[k];
				if (M->blk_of[j] == b)
					a[r * s + loc[j]] += M->val[k];
			}
		}
		/* dense LU with partial pivoting: P A = L U, L unit lower */
		int *piv = M->piv + b0;
		for (int k = 0; k < s; k++) {
			int p = k;
			double amax = fabs(a[k * s + k]);
			for (int r = k + 1; r < s; r++)
				if (fabs(a[r * s + k]) > amax) {
					amax = fabs(a[r * s + k]);
					p = r;
				}
			piv[k] = p;
			if (p != k)
				for (int c = 0; c < s; c++) {
					double t = a[k * s + c];
					a[k * s + c] = a[p * s + c];
					a[p * s + c] = t;
				}
			assert(a[k * s + k] != 0.);
			double inv = 1. / a[k * s + k];
			for (int r = k + 1; r < s; r++) {
				double l = a[r * s + k] * inv;
				a[r * s + k] = l;
				if (l != 0.)
					for (int c = k + 1; c < s; c++)
						a[r * s + c] -= l * a[k * s + c];
			}
		}
	}
	free(loc);
	M->has_lu = 1;
}

void sparse_solve(gdn_sparse *M, gdn_real *rhs)
{
	assert(M->has_lu);
	double *y = (double *)xmalloc(sizeof(double) * (M->max_blk ? M->max_blk : 1));
	for (int b = 0; b < M->nblk; b++) {
		const int b0 = M->blk_ptr[b];
		const int s = M->blk_ptr[b + 1] - b0;
		const double *a = M->lu + M->lu_ptr[b];
		const int *piv = M->piv + b0;
		for (int r = 0; r < s; r++) {
			int i = M->blk_idx[b0 + r];
			double acc = rhs[i];
			for (long long k = M->rp[i]; k < M->rp[i + 1]; k++) {
				int j = M->col[k];
				if (M->blk_of[j] != b)
					acc -= M->val[k] * rhs[j];
			}
			y[r] = acc;
		}
		for (int k = 0; k < s; k++)
			if (piv[k] != k) {
				double t = y[k];
				y[k] = y[piv[k]];
				y[piv[k]] = t;
			}
		for (int r = 1; r < s; r++) {
			double acc = y[r];
			for (int c = 0; c < r; c++)
				acc -= a[r * s + c] * y[c];
			y[r] = acc;
		}
		for (int r = s - 1; r >= 0; r--) {
			double acc = y[r];
			for (int c = r + 1; c < s; c++)
				acc -= a[r * s + c] * y[c];
			y[r] = acc / a[r * s + r];
		}
		for (int r = 0; r < s; r++)
			rhs[M->blk_idx[b0 + r]] = y[r];
	}
	free(y);
}

long long gdn_sparse_shim_nnz(const gdn_sparse *M)
{
	return M->has_csr ? M->rp[M->n] : M->coo_n;
}

int gdn_sparse_shim_max_block(const gdn_sparse *M)
{
	return M->max_blk;
}

int gdn_sparse_shim_nblocks(const gdn_sparse *M)
{
	return M->nblk;
}
