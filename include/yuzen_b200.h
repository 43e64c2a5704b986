/*
 * yuzen_b200.h -- the C ABI of the B200 implicit-step library.
 *
 * Plain pointers and sizes only.  Every entry point returns an int status:
 *    0  success (for a solve: converged)
 *    1  a solve hit its iteration limit
 *    2  a solve broke down or produced NaN
 *   -1  usage error (bad argument, wrong order of calls)
 *   -2  CUDA error
 * yz_last_error() describes the last non-zero status of the calling thread.
 * No exception crosses this boundary.  A context is used from one host
 * thread at a time and owns one CUDA stream and all its device buffers.
 *
 * ---------------------------------------------------------------------
 * Seam 1: the linear solve.  Replaces ILinearSolverBackend
 * (yuzen/src/numerics/LinearSolverBackend.h:56-103) and the factory entry
 * MakeLinearSolverBackend(name, inPlane) (LinearSolverBackend.h:130-131):
 * a maintainer adds the name "b200" to the factory and a thin adapter class
 * that forwards Build / Solve / Memory / SetMemory here (the adapter is
 * yuzen_b200/host/yz_backend_adapter.cpp).
 * ---------------------------------------------------------------------
 */
#ifndef YUZEN_B200_H
#define YUZEN_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct yz_solver yz_solver;

/* LinearSolverSettings (LinearSolverBackend.h:38-51); precondition uses the
 * values of tPrecondition: 0 None, 1 Jacobi, 2 ILU (ILU selects SA-AMG with
 * SPAI0 smoothing, as the reference's amgcl backend maps it). */
typedef struct yz_settings
{
	int    precondition;
	int    scaling;
	int    max_iteration;
	double epsilon;
	int    conc;
} yz_settings;

/* Which arithmetic the inner solve runs in. */
enum { YZ_PREC_FP64 = 0, YZ_PREC_FP32_REFINED = 1 };

const char* yz_last_error(void);

/* Create a solver context on a CUDA device (ILinearSolverBackend's
 * construction through MakeLinearSolverBackend, LinearSolverBackend.cpp:759). */
int yz_solver_create(int device, yz_solver** out);
int yz_solver_destroy(yz_solver* s);

/* ILinearSolverBackend::Build (LinearSolverBackend.h:66-72) plus the pattern,
 * which the reference fixes after the first assembly: row pointers (n+1), the
 * column-sorted mirror (CRS_Matrix::SortedColIndData, CRS_Matrix.h:247-251)
 * and the gather permutation (CRS_Matrix::SortedSrcData, CRS_Matrix.h:257),
 * host arrays.  May be called again when the pattern changes. */
int yz_solver_set_pattern(yz_solver* s, int n, int nnz, const int* rowptr,
                          const int* sorted_col, const int* sorted_src);

/* ILinearSolverBackend::Solve (LinearSolverBackend.h:74-88): values in the
 * storage order of the CRS (diagonal first in every row), host arrays; x is
 * the initial guess on entry and the solution on return (left untouched on a
 * breakdown, as the reference's amgcl backend leaves it).  iter and resid as
 * the reference reports them (relative residual). */
int yz_solver_solve(yz_solver* s, const yz_settings* set, const double* values,
                    const double* rhs, double* x, int* iter, double* resid);

/* The same on device pointers already resident on the context's device. */
int yz_solver_solve_device(yz_solver* s, const yz_settings* set, const double* d_values,
                           const double* d_rhs, double* d_x, int* iter, double* resid);

/* Inner-solve arithmetic (YZ_PREC_*).  FP64 is the drop-in parity path. */
int yz_solver_set_precision(yz_solver* s, int precision);

/* ILinearSolverBackend::Memory / SetMemory (LinearSolverBackend.h:89-102):
 * the TryBackoff counters.  yz_solver_memory returns the count written. */
int yz_solver_memory(const yz_solver* s, double* out, int cap);
int yz_solver_set_memory(yz_solver* s, const double* m, int len);

/* The AMG hierarchy of the last AMG-preconditioned solve, for structure
 * checks: number of levels; per level rows, nnz(A), nnz(P) and whether it is
 * the directly solved level; and copies of A_l, P_l and the aggregate map
 * into host buffers sized from yz_solver_level_info (null pointers skipped). */
int yz_solver_levels(const yz_solver* s);
int yz_solver_level_info(const yz_solver* s, int level, int* rows, int* nnz_a,
                         int* nnz_p, int* direct);
int yz_solver_level_copy(const yz_solver* s, int level, int* a_ptr, int* a_col,
                         double* a_val, int* p_ptr, int* p_col, double* p_val, int* agg);

/* Timing of the last solve on the context's stream (CUDA events):
 * milliseconds in AMG set-up and in the Krylov iterations. */
int yz_solver_last_timing(const yz_solver* s, double* setup_ms, double* iterate_ms);

/* Kernels this context launched since creation (a launch counter kept by the
 * host side of the library). */
long long yz_solver_launches(const yz_solver* s);

/* Building blocks exposed for the parity tests: the deterministic dot
 * product every reduction of the solve uses, and CRS_Matrix::MatVec
 * (CRS_Matrix.cpp:307-329), on host arrays through the device. */
int yz_dot(int n, const double* x, const double* y, double* out);
int yz_spmv(int n, int nnz, const int* rowptr, const int* col, const double* val,
            const double* x, double* y);

#ifdef __cplusplus
}
#endif

#endif
