/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * Stand-in for the reference's sparse operator header (src/maths/sparse.h).
 * The reference implements these entry points on top of SuiteSparse CXSparse
 * and KLU, neither of which is installed here.  When the reference's own
 * sources (src/dg, src/simulation, src/mesh, src/models) are compiled in place
 * for the oracle, this directory is put first on the include path so that
 * `#include <maths/sparse.h>` resolves to this file.  The prototypes are the
 * reference's (src/maths/sparse.h:42-77, same names, argument meaning and
 * in-place conventions); the type `gdn_sparse` is our own and opaque to the
 * reference code, which never touches its fields.  The implementation in
 * ../sparse_shim.c is written from the mathematics (COO accumulation, CSR with
 * summed duplicates, SpMV, SpGEMM, alpha*A+beta*B, and a direct solve by
 * strongly-connected-block triangular ordering with dense LU per block).
 */
#ifndef GDN_ORACLE_SPARSE_SHIM_H
#define GDN_ORACLE_SPARSE_SHIM_H

#include <stdbool.h>
/* The reference header pulls these in through cs.h / klu.h; files that include
 * <maths/sparse.h> rely on them (NULL, stdout, malloc, ...). */
#include <limits.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <gdon3d.h>

typedef struct gdn_sparse gdn_sparse;

gdn_sparse *gdn_sparse_malloc();
gdn_sparse *sparse_coo_init(int n);
gdn_sparse *sparse_coo_init_identity(int n);
gdn_sparse *sparse_init_copy(gdn_sparse *M);
void sparse_free(gdn_sparse *M);
void gdn_sparse_coo_switch_on(gdn_sparse *M, int i, int j);
void sparse_coo_insert(gdn_sparse *M, int i, int j, gdn_real val);
void sparse_csr_allocate(gdn_sparse *M, bool free_coo);
void sparse_csr_add_entry(gdn_sparse *M, int i, int j, gdn_real val);
void sparse_csr_set_entry(gdn_sparse *M, int i, int j, gdn_real val);
gdn_real sparse_csr_get_entry(gdn_sparse *M, int i, int j);
gdn_sparse *sparse_csr_matrix_multiplication(const gdn_sparse *A,
                                             const gdn_sparse *B);
gdn_sparse *sparse_csr_matrix_addition(const gdn_sparse *A, const gdn_sparse *B,
                                       const gdn_real alpha,
                                       const gdn_real beta);
void sparse_spmdv(const gdn_sparse *A, const gdn_real *x, gdn_real *res);
void sparse_solver_init(gdn_sparse *A);
void sparse_solver_lu_factor(gdn_sparse *M);
void sparse_solve(gdn_sparse *A, gdn_real *rhs);

/* Shim-only diagnostics (not in the reference API). */
long long gdn_sparse_shim_nnz(const gdn_sparse *M);
int gdn_sparse_shim_max_block(const gdn_sparse *M);
int gdn_sparse_shim_nblocks(const gdn_sparse *M);

#endif
