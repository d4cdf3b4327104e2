/* Host symbolic analysis for the supernodal Cholesky of a sparse SPD matrix.
 *
 * Replaces the analysis half of cholmod_l_analyze (called from
 * src/speigs_core.c:934 of the reference, with AMD or METIS chosen at
 * :859-863): a fill-reducing ordering, the elimination tree, column counts,
 * supernode partition with relaxed amalgamation, the row structure of every
 * supernode and the relative index maps used by the multifrontal
 * extend-add.  Everything here is host integer work done once per call; the
 * numeric factorization and the solves run on the device.
 *
 * Conventions: all indices after ordering are in the NEW numbering.  The
 * input is the full symmetric pattern (both triangles, CSR == CSC).
 */
#ifndef SPX_SYMBOLIC_H
#define SPX_SYMBOLIC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spx_symbolic {
    int32_t  n;
    int32_t  nsuper;
    int32_t *perm;        /* [n]   perm[new] = old                             */
    int32_t *iperm;       /* [n]   iperm[old] = new                            */
    int32_t *sfirst;      /* [nsuper+1] supernode s owns columns [sfirst[s], sfirst[s+1]) */
    int32_t *sparent;     /* [nsuper] parent supernode, -1 for a root          */
    int64_t *rowptr;      /* [nsuper+1] offsets into rows / relmap             */
    int32_t *rows;        /* row list of each supernode: its own c columns first,
                             then the rows below, ascending                      */
    int32_t *relmap;      /* same indexing as rows; for a below row (t >= c) the
                             position of that row in the parent's row list      */
    int64_t *frontptr;    /* [nsuper+1] offsets of the r x r column-major fronts */
    int32_t *col2sup;     /* [n]   supernode owning each column                */
    int32_t  nlevels;
    int32_t *level_ptr;   /* [nlevels+1] supernodes grouped by tree level      */
    int32_t *level_sup;   /* [nsuper] leaves first (level 0), roots last       */
    int32_t *child_ptr;   /* [nsuper+1] children lists                          */
    int32_t *child_list;  /* [nsuper]                                           */
    int64_t  nnzL;        /* entries of L (lower triangle incl. diagonal)      */
    int64_t  front_total; /* sum of r*r                                         */
    double   flops;       /* factorization flops (POTRF+TRSM+SYRK, counted as in LAPACK) */
    int32_t  max_rows;    /* largest r                                          */
    int32_t  max_cols;    /* largest c                                          */
} spx_symbolic;

/* Ordering methods. */
#define SPX_ORDER_AUTO     0
#define SPX_ORDER_MINDEG   1   /* stands where the reference asks for AMD   */
#define SPX_ORDER_ND       2   /* stands where the reference asks for METIS */

/* Analyse the pattern of a symmetric matrix given in full CSR (both
 * triangles; the diagonal may or may not be present).  Returns 0 on success,
 * -2 on allocation failure, -1 on bad input. */
int spx_analyze(int32_t n, const int64_t *rowptr, const int32_t *col,
                int ordering, spx_symbolic *S);

void spx_symbolic_free(spx_symbolic *S);

/* Fill-reducing ordering alone (perm[new] = old).  Exposed for tests. */
int spx_order(int32_t n, const int64_t *rowptr, const int32_t *col,
              int ordering, int32_t *perm);

#ifdef __cplusplus
}
#endif
#endif
