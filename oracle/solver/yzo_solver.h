/*
 * yzo_solver.h -- the CPU oracle of the linear solve (TEST INFRASTRUCTURE).
 *
 * This is the checker the CUDA solver in yuzen_b200/ is compared against; it
 * is never part of the product path. It restates, on plain arrays, the two
 * backends of the reference's solver seam:
 *
 *   flavour YZO_AMG   -- AmgclBackend::Solve, LinearSolverBackend.cpp:539-728:
 *                        BiCGStab preconditioned by smoothed-aggregation AMG
 *                        with SPAI0 smoothing (ILU), damped Jacobi (None /
 *                        Jacobi), SPAI0 tried first on a concentration solve
 *                        (opt concpc) with the TryBackoff of :262-270, and
 *                        coarse_enough 500 on systems above 3000 rows
 *                        (opt amgcoarse, :660-675).
 *   flavour YZO_ILU0  -- EigenBackend::Solve, LinearSolverBackend.cpp:370-463,
 *                        restated with ILU(0) in place of Eigen's ILUT (fill
 *                        10, droptol 1e-10) and without the block-ILUT try.
 *
 * AMGCL 1.4.4 and Eigen 3.4.0 are not available here, so bit parity to those
 * libraries is UNPINNED. The algorithms are written from their published
 * descriptions (van der Vorst 1992; Vanek, Mandel, Brezina 1996; Broeker and
 * Grote 2002) with AMGCL's documented defaults, and every floating-point
 * operation is specified so that the CUDA solver can reproduce it exactly:
 * see yzo_solver.cpp for the definitions (reduction tree, MIS-2 aggregation,
 * Galerkin product summation order, Gauss-Jordan coarse inverse).
 */
#ifndef YZO_SOLVER_H
#define YZO_SOLVER_H

#ifdef __cplusplus
extern "C" {
#endif

enum { YZO_AMG = 0, YZO_ILU0 = 1 };
/* LinearSolverSettings::tPrecondition, LinearSolverBackend.h:40 */
enum { YZO_PC_NONE = 0, YZO_PC_JACOBI = 1, YZO_PC_ILU = 2 };

typedef struct yzo_settings
{
	int    precondition;   /* YZO_PC_* */
	int    scaling;        /* divide each row by its diagonal */
	int    max_iteration;
	double epsilon;        /* relative residual tolerance */
	int    conc;           /* the solver of a concentration equation */
} yzo_settings;

typedef struct yzo_solver yzo_solver;

yzo_solver* yzo_create(int flavour);
void        yzo_destroy(yzo_solver* s);

/*
 * Solve A x = rhs.  The matrix is given as the reference's CRS_Matrix hands
 * it to a backend: row pointers, the column-sorted mirror (sorted_col) and the
 * permutation sorted_src that picks the k-th sorted value out of values[]
 * (storage order, diagonal first in every row: CRS_Matrix.h:59-68).
 * x is in/out: the initial guess on entry.  Returns 0 converged, 1 iteration
 * limit, 2 breakdown / NaN (LinearSolverBackend.h:74-88).
 */
int yzo_solve(yzo_solver* s, const yzo_settings* set, int n,
              const int* rowptr, const int* sorted_col, const int* sorted_src,
              const double* values, const double* rhs, double* x,
              int* iter, double* resid);

/* The fault switch of LinearSolverBackend.cpp:630-645 (also read from
 * YUZEN_FAULT_AMGCL=k:m at the first solve): solves at .. at+count-1 of the
 * process that reach the AMG / Jacobi path break down before iterating;
 * at = 0 switches it off.  Resets the process's solve count. */
void yzo_fault_inject(long at, long count);

/* TryBackoff counters (ILinearSolverBackend::Memory / SetMemory). */
int  yzo_memory(const yzo_solver* s, double* out, int cap);
void yzo_set_memory(yzo_solver* s, const double* m, int len);

/*
 * The AMG hierarchy of the last ILU-preconditioned AMG solve.
 * yzo_levels: number of levels (the last one is the coarsest).
 * yzo_level_info: rows, nnz of A_l, nnz of P_l (0 on the last level),
 *                 and whether the level is solved directly.
 * yzo_level_copy: copies the CSR of A_l (ptr, col, val) and of P_l
 *                 (ptr, col, val) into caller buffers sized from level_info
 *                 (any pointer may be null); agg receives the aggregate of
 *                 every row (-1 for a row left out).
 */
int yzo_levels(const yzo_solver* s);
int yzo_level_info(const yzo_solver* s, int l, int* rows, int* nnzA, int* nnzP, int* direct);
int yzo_level_copy(const yzo_solver* s, int l, int* aptr, int* acol, double* aval,
                   int* pptr, int* pcol, double* pval, int* agg);

/* The deterministic dot product every reduction of the solve uses. */
double yzo_dot(int n, const double* x, const double* y);

/* CRS_Matrix::MatVec restated: y_i summed in the given order from 0. */
void yzo_spmv(int n, const int* rowptr, const int* col, const double* val,
              const double* x, double* y);

#ifdef __cplusplus
}
#endif

#endif
