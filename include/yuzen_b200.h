/*
 * yuzen_b200.h -- the C ABI of the B200 implicit-step library.
 *
 * Plain pointers and sizes only.  Every entry point returns an int status:
 *    0  success (for a solve: converged)
 *    1  a solve hit its iteration limit
 *    2  a solve broke down or produced NaN
 *   -1  usage error (bad argument, wrong order of calls)
 *   -2  CUDA error
 *   -3  the time step failed numerically (yz_step_advance only): dt fell
 *       below MinDt, or the Newton iteration did not converge at a fixed
 *       step -- the cases where the reference aborts with FatalError
 *       (ImplicitSolver.cpp:180-184, :192-201); the message is the
 *       reference's.  The step context is then left mid-step (its dt and
 *       Newton guess changed): restore it with yz_step_set_fields (or
 *       yz_step_set_state) before advancing it again.
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

/* Which arithmetic the AMG preconditioner runs in.  YZ_PREC_FP64: all of it
 * (the drop-in parity path).  YZ_PREC_FP32_CYCLE: the set-up in FP64 as
 * always, then every level's A, SPAI0 diagonal, P, R and the coarsest
 * inverse rounded to float, and the V-cycle run in float; the BiCGStab
 * around it (its SpMVs, dot products, residuals, convergence test and the
 * solution) stays FP64, so a converged solve meets the same tolerance.
 * YZ_PREC_FP32_MATRIX: the same cycle, and the BiCGStab's SpMVs read the
 * matrix rounded to float (vectors, dot products, recurrences and the test
 * FP64): the solve meets its tolerance on the rounded matrix, a relative
 * change of the system of about 6e-8, which the Newton iteration's FP64
 * residual corrects in the step. */
enum { YZ_PREC_FP64 = 0, YZ_PREC_FP32_CYCLE = 1, YZ_PREC_FP32_MATRIX = 2 };

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

/* Preconditioner arithmetic (YZ_PREC_*), from the next solve on. */
int yz_solver_set_precision(yz_solver* s, int precision);

/* AMG hierarchy reuse.  0 (the default, the reference's way): a new SA-AMG
 * set-up for every solve.  k > 0: a set-up serves up to k further solves of
 * the same pattern -- the finest level's SPAI0 is recomputed from each new
 * matrix and the cycle's finest level is the new matrix, the coarser levels
 * are the set-up's -- and the BiCGStab loop is replayed as one cached CUDA
 * graph.  A solve on a reused hierarchy that fails is repeated on a new
 * set-up; one that takes clearly more iterations than the set-up's first
 * solve (more than max(4, half) again) makes the next solve set up afresh.
 * The Krylov solve stays FP64 to the same tolerance. */
int yz_solver_set_amg_reuse(yz_solver* s, int max_solves);

/* The BiCGStab loop as one CUDA graph launch per solve (1, the default) or
 * launched from the stream with one iteration in flight (0).  The graph is
 * captured from the context's stream in thread-local capture mode, so other
 * host threads may drive their own contexts (and allocate) meanwhile. */
int yz_solver_set_graph_loop(yz_solver* s, int on);

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
/* Kernels the library launched in this process, all contexts. */
long long yz_launch_count(void);
/* Time every later launch of the kernel with this name (its function name in
 * the library, e.g. "KSpmvAlpha"; null or "" stops) with CUDA events on the
 * stream it is launched on, and clear what was collected. */
int yz_time_kernel(const char* name);
/* Device time summed over the timed launches, and their count. */
int yz_kernel_time(double* total_ms, long long* launches);

/* Fault injection, the test switch of the reference's amgcl backend
 * (LinearSolverBackend.cpp:630-645, environment YUZEN_FAULT_AMGCL=k:m, which
 * this library reads too): `count` solves of the process, from the at-th of
 * those that reach the SA-AMG or Jacobi path on, break down before they
 * iterate -- return 2, x left as given, unless x already meets the
 * tolerance -- so that a step cuts dt and retries (or, at a fixed step,
 * fails with -3).  at = 0 switches it off; the call restarts the count. */
int yz_fault_inject(long long at, long long count);

/* The reference's profile table (util/Profile.h: YUZEN_PROF scopes, switched
 * on by the environment variable YUZEN_PROFILE, totals to standard error at
 * exit as "[profile] name calls seconds").  The device path keeps the names
 * (step, h.assemble, h.couple, h.linsolve, h.after, c.linsolve, lin.prepare,
 * lin.precond, lin.iterate, lin.fallback.conc, lin.learned), the switch and
 * the exit lines; a scope's seconds are the device time of the work it
 * queued on its stream (CUDA events), and every scope is an NVTX range of
 * its name whether the switch is on or not.  yz_profile_entry gives the
 * index-th name's totals so far (returns 1 past the last name, 0 otherwise;
 * the name stays valid until the next call); yz_profile_reset zeroes them;
 * yz_profile_enabled is 1 with the switch on. */
int yz_profile_enabled(void);
int yz_profile_entry(int index, const char** name, long long* calls, double* seconds);
int yz_profile_reset(void);

/* Building blocks exposed for the parity tests: the deterministic dot
 * product every reduction of the solve uses, and CRS_Matrix::MatVec
 * (CRS_Matrix.cpp:307-329), on host arrays through the device. */
int yz_dot(int n, const double* x, const double* y, double* out);
int yz_spmv(int n, int nnz, const int* rowptr, const int* col, const double* val,
            const double* x, double* y);

/* The dot product of yz_dot for callers that cannot allocate device memory
 * (a host code that owns all device memory itself, or a path that must not
 * take cudaMalloc's device-wide synchronisation).  This entry point has no
 * counterpart in the reference.  d_x, d_y (n each) and d_out (one double) are
 * the caller's device arrays on the current device; the call is queued on
 * `stream` (a cudaStream_t, null: the default stream) and allocates nothing:
 * its scratch is a static array of the library, at most
 * yz_dot_noalloc_max() elements (16,777,216); larger n returns -1.  The
 * array is shared by every call, so calls that overlap on the GPU race; the
 * first call on a device takes the array's address (cudaGetSymbolAddress)
 * and should come before any stream capture.  That address is kept per
 * device index for the life of the process and belongs to the device's
 * primary context: after cudaDeviceReset, or from a thread whose current
 * context is a non-primary driver context, the kept address is stale and
 * the call must not be used. */
int yz_dot_noalloc(int n, const double* d_x, const double* d_y, double* d_out, void* stream);
long long yz_dot_noalloc_max(void);

/*
 * ---------------------------------------------------------------------
 * Seam 2: the whole implicit step of the well-mixed film-height equation.
 * Replaces C_NewtonKantorovich::TimeAdvance (NewtonKantorovich.cpp:424-486)
 * with the hooks of WellMixed_HeightEquationBase (HeightEquationBase.h:
 * SetMatrixA :670-788, ApplyA :804-827, SetMatrixJacobi :1062-1091,
 * BeforeNKLoop / EveryNKLoop / AfterNKLoop :1314-) and the clock advance of
 * the model loop (WellMixedModelBase.h:1334, TimeSteps.cpp:121-160), on a 2-D
 * grid with two ghost layers (nx = Nx+4, row of cell (ix,iy) = iy*nx + ix,
 * Grids.h:256).  Everything is non-dimensional, as the reference's model
 * holds it after NonDimensionalNumbers::Build (NonDimensionalNumbers.cpp:43).
 * ---------------------------------------------------------------------
 */
typedef struct yz_step yz_step;

/* BoundaryCondition::tBoundaryCondition (BoundaryCondition.h:56-63).  The
 * film takes every kind (ghost rows as BoundaryCondition2D::Apply writes
 * them, BoundaryCondition.cpp:104-187, 376-517; a Pinning corner next to a
 * FreshInlet or an Outlet edge, and two Pinning edges meeting, are refused
 * as the reference refuses or leaves them), for the film and for the
 * concentration equation (conc_field) alike. */
enum { YZ_BC_SYMMETRY = 0, YZ_BC_PERIODIC = 1, YZ_BC_PINNING = 2, YZ_BC_FRESHINLET = 3, YZ_BC_OUTLET = 4 };

/* C_Interpolation_base4::t_Scheme (FiniteDifferences.h:42-53), the face
 * interpolation of Numerics.Convection.Height / .Concentration: the
 * limited ones (Koren, the height's default, and VanLeer) and the fixed
 * four-point ones, for both. */
enum { YZ_SCHEME_UPWIND1 = 0, YZ_SCHEME_UPWIND2 = 1, YZ_SCHEME_CENTRAL2 = 2, YZ_SCHEME_UTOPIA = 3,
       YZ_SCHEME_QUICK = 4, YZ_SCHEME_KK = 5, YZ_SCHEME_CENTRAL4 = 6, YZ_SCHEME_KOREN = 7,
       YZ_SCHEME_VANLEER = 8 };

typedef struct yz_step_params
{
	int    nx, ny;                /* points including the ghost layers */
	int    bc[4];                 /* Xmin, Xmax, Ymin, Ymax */
	double dx, dy;                /* C_Grid2D spacing */
	double xmin, ymin;            /* the grid's lower corner: X / Y of the low faces of cell (0,0) (RectGrid.h:375-383) */
	double theta;                 /* 0.5: Crank-Nicolson */
	/* physics terms (HeightEquationBase.h:565-577) */
	int    on_laplace, on_vgrav, on_pgrav, on_marangoni, on_centrifugal, on_disjoining;
	int    on_evap, conc_field;   /* conc_field 0: c carried unchanged (Physics.ConcField = None) */
	double Bo, Dp, hstar, disj_n, disj_m, lambda_slip, Ev;
	/* property laws (FluidProperty.h:100-181) */
	double visc_c0, visc_base, visc_exp;
	double sig_c0, sig_base, sig_coef;
	/* evaporation (Evaporation.cpp), non-dimensional with Coef = 1 */
	int    ev_conc_func;          /* 0 Raoult, 1 PowerN */
	int    ev_spatial;            /* 0 uniform, 1 negPow */
	int    ev_hast_modify;
	double ev_m_resin, ev_m_solvent, ev_power_n, ev_conc_r, ev_negpow_exp, ev_negpow_rmax, ev_h_ast;
	/* Newton-Kantorovich (NewtonKantorovich.h:56-70) */
	int    nk_max, nk_min;
	double nk_eps, nk_eps_rel;
	/* the linear solve of the height equation */
	yz_settings lin;
	/* time-step control (ImplicitSolver.cpp:144-190, 271-307) */
	int    dt_control, dt_keep_steps;
	double dt, dt_max, dt_min, dt_change_factor, dt_criterion, dt_scale_floor;
	double t_start;
	/* the upwinded terms (BodyForceKernel.h, ParallelGravityKernel.h,
	 * CentrifugalKernel.h, SolutoCapillarityKernel.h) */
	int    conv_height;           /* any YZ_SCHEME_* (Koren is the reference's default) */
	double Pgx, Pgy;              /* in-plane gravity groups (coefficients Pg/3) */
	double Sp, rot_x, rot_y;      /* rotation group and the axis (non-dimensional) */
	double As, Ma;                /* Marangoni coefficient As*Ma/2 */
	/* the well-mixed concentration equation (ConcEquationBase.h), solved in
	 * every Newton pass when conc_field = 1 */
	int    conv_conc;             /* any YZ_SCHEME_* (UTOPIA is the reference's default) */
	int    conc_convection, conc_diffusion;
	double theta_c;               /* 0.5 (Crank-Nicolson) */
	double Df, diff_c0, diff_base, diff_exp;   /* Df and the diffusivity law D(c) = base exp(exp (c - c0)) */
	yz_settings lin_conc;         /* its linear solve (conc = 1: the SPAI0-first role) */
	/* the liquid supply of a nozzle (Physics.Source; SourceBase.cpp,
	 * WM2D/Source.cpp): flow rate src_rate (1 - exp(-t / src_tau)) into the
	 * cells' area fractions within src_radius of the nozzle, sampled on
	 * src_subregions^2 points a cell; the nozzle at the tip of an arm of
	 * length src_arm about (src_arm_x, src_arm_y) turning at src_omega from
	 * src_angle0, its angular speed ramped up over src_ramp, held over
	 * src_plateau and ramped down, from src_t0; evaluated at the middle of
	 * each step.  With conc_field the supplied liquid arrives at src_conc
	 * (src_supplied = 1, ConcType "supplied") or at the local c (0). */
	int    on_source, src_subregions;
	double src_radius, src_rate, src_tau, src_arm, src_arm_x, src_arm_y, src_omega, src_angle0, src_ramp,
	       src_plateau, src_t0;
	int    src_supplied;
	double src_conc;
} yz_step_params;

typedef struct yz_step_stats
{
	int    steps;              /* steps taken by this call */
	int    newton_iterations;  /* Newton passes, summed */
	int    linear_iterations;  /* BiCGStab iterations, summed */
	int    retries;            /* attempts cut and repeated (dt control) */
	double time;               /* the clock after the call */
	double dt;                 /* DT().now after the call */
	double last_resid;         /* Newton correction of the last pass */
	double setup_ms, solve_ms, assemble_ms;  /* device time in AMG set-up, Krylov iterations, assembly */
	double device_ms;          /* the whole call on the step's stream (CUDA events) */
	long long launches;        /* kernels the call launched */
	int    conc_iterations;    /* BiCGStab iterations of the concentration solves, summed */
	int    conc_solves;        /* concentration solves */
	/* with the energy history on (yz_step_set_energy): after the call, the
	 * free energy and flux power of the film, the energy dissipated since
	 * the history started and the balance of the last step
	 * (WellMixedModelBase.h:1405-1411); 0 otherwise */
	double energy_F, energy_D, energy_dissipated, energy_balance;
	int    amg_setups;         /* SA-AMG hierarchies set up (height and concentration solves) */
	/* the learned preconditioner (yz_step_set_learned), for this call: film
	 * solves it converged, solves it handed back to SA-AMG, its BiCGStab
	 * iterations, the samples held, the device time spent training, and the
	 * network's held-out error against the V-cycle and last training loss
	 * (-1 before it is trained) */
	int    learned_solves, learned_fallbacks, learned_iterations, learned_samples;
	double learned_train_ms, learned_val_err, learned_loss;
} yz_step_stats;

/* Build the step: fields h, c, s on all nx*ny points (host arrays). */
int yz_step_create(int device, const yz_step_params* p, const double* h, const double* c,
                   const double* s, yz_step** out);
int yz_step_destroy(yz_step* st);
/* Preconditioner arithmetic (YZ_PREC_*) of the step's height and
 * concentration solves, from the next solve on; FP64 unless set. */
int yz_step_set_precision(yz_step* st, int precision);
/* The energy history (Output.Energy): on = 1 evaluates the budget of the
 * present film (yz_step_energy) and starts the dissipated energy at 0; every
 * later step evaluates it at the film it ends on and adds the step's
 * Crank-Nicolson share of the flux power (WellMixedModelBase.h:1405-1411). */
int yz_step_set_energy(yz_step* st, int on);
/* AMG hierarchy reuse (yz_solver_set_amg_reuse) for the step's solves. */
int yz_step_set_amg_reuse(yz_step* st, int max_solves);
/* The graph form of the step's BiCGStab loops (yz_solver_set_graph_loop). */
int yz_step_set_graph_loop(yz_step* st, int on);

/* The FP32 V-cycle's shape, for one context (both of a step's solvers):
 * fuse_from the first level whose way down and way up run as one launch
 * each (-1: the library's default, level 2 or YZ_FUSE_FROM; 0: none),
 * coarse_lanes the lanes a row of the coarse levels' kernels (0: by the
 * level's mean row length; 1, 2, 4 or 8), fine_sweeps the post-smoothing
 * sweeps at the finest level (0: the default, 5 or YZ_FINE_SWEEPS; 1 to 8).
 * The launch shapes change the preconditioner by float rounding only, the
 * sweeps change it (a better one); the FP64 cycle, the reference's, is not
 * affected.  yuzen_b200.autotune picks them per instance size. */
int yz_solver_set_tuning(yz_solver* s, int fuse_from, int coarse_lanes, int fine_sweeps);
int yz_step_set_tuning(yz_step* st, int fuse_from, int coarse_lanes, int fine_sweeps);
/* The energy budget of the film the step holds (WellMixed_ModelBase::EnergyEval,
 * WellMixedModelBase.h:883-893, after EnergyBudget.h): the free energy F and
 * the flux power D (HeightEquationBase::FluxPower), both times the cell
 * measure. */
int yz_step_energy(yz_step* st, double* F, double* D);
/* Advance nsteps time steps (TimeAdvance + the clock advance each). */
int yz_step_advance(yz_step* st, int nsteps, yz_step_stats* stats);
/* Fields after the last step (host arrays of nx*ny; null pointers skipped). */
int yz_step_get_fields(yz_step* st, double* h, double* c);
/* Replace the committed fields (host arrays of nx*ny; null pointers skipped):
 * the film the next step starts from, as C_ImplicitSolver::SetX takes it
 * (phi_old = phi_new = h, ImplicitSolver.cpp:94-101). */
int yz_step_set_fields(yz_step* st, const double* h, const double* c);
/* The state a later step depends on (the reference's RestartState,
 * IO/RestartState.h:57): the film and concentration, phi_old, phi_old2,
 * phi_new, the last Newton correction (the next solve's guess), the clock
 * and its controller, the Eisenstat-Walker and extrapolation memory, the
 * solvers' TryBackoff counters and the energy history, as
 * yz_step_state_size() doubles.  A step given a state with yz_step_set_state
 * continues as the step it was taken from would have, bit for bit on the
 * FP64 path (an AMG hierarchy kept for reuse is not part of the state: the
 * next solve of a reuse form sets one up). */
long long yz_step_state_size(const yz_step* st);
int yz_step_get_state(yz_step* st, double* out);
int yz_step_set_state(yz_step* st, const double* in, long long len);
/* The fixed CRS pattern of A / I + theta dt J, storage order (diagonal
 * first): rowptr n+1, col nnz, boundary flags n.  nnz is returned. */
int yz_step_pattern(yz_step* st, int* rowptr, int* col, int* bc);
/* One Newton pass's system at the film h (as SetMatrixA, SetMatrixJacobi,
 * MakeMatrix_IA, ApplyA and MakeRHS build it with phi_old, phi_guess = h and
 * the explicit half A(h_old) h_old, evaporation at h_old): values of
 * I + theta dt J (nnz, storage order) and the right-hand side (n). */
int yz_step_system(yz_step* st, const double* h_old, const double* h, double dt,
                   double* ia_values, double* rhs);
/* The concentration equation's pattern (conc_field = 1): rowptr n+1 and col
 * (storage order, diagonal first, ConcEquationBase.h:243-259); nnz is
 * returned, 0 without the concentration equation. */
int yz_step_conc_pattern(yz_step* st, int* rowptr, int* col);
/* The concentration system of the first Newton pass of a step that starts
 * from the committed film h and concentration c (ConcEquationBase.h:271-396
 * with h1 = h0 = h, the face fluxes F1 = F0 at that film, the limiter at c):
 * the matrix values (storage order) and the right-hand side of the
 * correction d = c1 - c0. */
int yz_step_conc_system(yz_step* st, const double* h, const double* c, double dt,
                        double* values, double* rhs);
/* The same pattern built on the host alone, without a device (the structure
 * C_ImplicitSolver::Alloc fixes, ImplicitSolver.cpp:60-81, with the ghost rows
 * of BoundaryCondition2D::Apply, BoundaryCondition.cpp:376-517); arrays may be
 * null to query nnz (the return value). */
int yz_pattern_2d(const yz_step_params* p, int* rowptr, int* col, int* bc);

/*
 * ---------------------------------------------------------------------
 * The learned preconditioner.  The reference has no counterpart: these
 * entry points add a preconditioner beside its SA-AMG one, for the film's
 * solve (LinearSolverBackend.cpp:660-679 is the AMG it sits beside and falls
 * back to).  A small U-Net on the film's grid (levels of 16, 32, 64 and 64
 * channels, 3x3 convolutions in BF16 on the tensor cores with FP32
 * accumulation) maps a residual r -- its input channels are r and r times
 * two feature maps, the matrix diagonal's and the film height's, and their
 * squares and product -- to z ~ V r, the SA-AMG V-cycle's answer; without
 * activation (activation 0, the preconditioner's form: no bias, no ReLU) it
 * is a linear operator on r whose coefficients follow the system;
 * it is trained on the device, by its own forward and backward kernels, on
 * (r, V r) pairs the solver collects from its own AMG-preconditioned solves,
 * and used in a flexible BiCGStab (the right-preconditioned iteration with a
 * preconditioner that may change between applications).  SA-AMG stays the
 * yardstick and the fallback: a learned solve that needs more than cap_factor
 * times the iterations of the last SA-AMG solve is repeated on the AMG path,
 * and the network then sits out a growing number of solves.
 * ---------------------------------------------------------------------
 */
typedef struct yz_unet yz_unet;

/* A network for a grid of nx x ny points (rows iy*nx + ix, ghost layers
 * included), holding up to `capacity` training pairs; weights initialised
 * from `seed`; activation 0 linear (no bias, no ReLU), 1 bias and ReLU. */
int yz_unet_create(int device, int nx, int ny, int capacity, unsigned seed, int activation, yz_unet** out);
int yz_unet_destroy(yz_unet* u);
long long yz_unet_param_count(const yz_unet* u);
/* The FP32 master weights (yz_unet_param_count floats). */
int yz_unet_get_params(yz_unet* u, float* out);
int yz_unet_set_params(yz_unet* u, const float* in);
/* The network's output for normalised input maps feat3 = [r/rms; diagonal
 * feature; height feature] (3 x n floats), in units of z / rms(r) (n floats). */
int yz_unet_forward(yz_unet* u, const float* feat3, float* out);
/* One pair's loss, sum over the n rows of (out - target)^2 / n, and its
 * gradient w.r.t. every weight (yz_unet_param_count floats). */
int yz_unet_loss_grad(yz_unet* u, const float* feat3, const float* target, double* loss, float* grad);
/* A training pair from host arrays: the residual r, the V-cycle's answer z,
 * the matrix diagonal and the film height (null: none), n each. */
int yz_unet_add_sample(yz_unet* u, const double* r, const double* z, const double* diag, const double* h);
int yz_unet_samples(const yz_unet* u);
/* Slot k (0 <= k < yz_unet_samples) of the pair ring, 4 x n floats: r/rms(r),
 * z/rms(r) and the two feature maps the pair was stored with (the diagonal's
 * log10|a_ii| / 4 and the film's log10 h / 2 + 1, 0 without a film); *valid 0
 * for a slot marked unused. */
int yz_unet_get_sample(yz_unet* u, int k, float* out, int* valid);
/* Adam over the pairs held, the last `holdout` kept out: iters steps of
 * `batch` pairs at learning rate lr; the last step's mean loss, and the
 * held-out relative error ||N r - V r|| / ||V r|| (-1 without held-out pairs). */
int yz_unet_train(yz_unet* u, int iters, int batch, float lr, int holdout, double* loss, double* val_err);
/* The network applied to a device vector r (n doubles) as the preconditioner
 * applies it: z = N(r), with the diagonal of d_values (storage order,
 * diagonal first in each row of d_rowptr) and the height d_h as features.
 * Queued on `stream` (a cudaStream_t, null: the default stream). */
int yz_unet_apply(yz_unet* u, const double* d_values, const int* d_rowptr, const double* d_h,
                  const double* d_r, double* d_z, void* stream);

/* The seam-1 solver with the network: mode 0 off; 1 collect (the next
 * `collect_solves` SA-AMG solves each add up to `per_solve` (r, V r) pairs to
 * the network's ring); 2 use (the flexible BiCGStab with the network first,
 * SA-AMG the fallback).  The network must be trained before mode 2 uses it
 * and must outlive its use by the solver. */
int yz_solver_set_learned(yz_solver* s, yz_unet* u, int mode, int collect_solves, int per_solve,
                          double cap_factor);
/* The film height (device vector of n) the network reads as a feature, for
 * the next solves; null: none. */
int yz_solver_set_aux(yz_solver* s, const double* d_h);
/* Counters of the learned path: solves it converged, fallbacks to SA-AMG,
 * its iterations, solves it sat out. */
int yz_solver_learned_stats(const yz_solver* s, int* solves, int* fallbacks, int* iterations, int* skipped);

/* The step's film solves with a learned preconditioner of its own: the
 * first `collect_solves` SA-AMG solves collect up to `samples_per_solve`
 * pairs each; the film solve after them trains the network (train_iters Adam
 * steps of `batch` pairs at rate lr, `holdout` pairs kept out to measure it
 * against the V-cycle); from then on every film solve tries the network
 * first, within cap_factor x the last SA-AMG solve's iterations.  The
 * concentration's solves keep their SPAI0 / SA-AMG path.  Null: off. */
typedef struct yz_learned_cfg
{
	int      collect_solves;
	int      samples_per_solve;
	int      capacity;
	int      train_iters;
	int      batch;
	float    lr;
	int      holdout;
	double   cap_factor;
	unsigned seed;
	int      activation;   /* 0 linear (the default), 1 ReLU */
} yz_learned_cfg;
int yz_step_set_learned(yz_step* st, const yz_learned_cfg* cfg);

/* One 3x3 convolution of the network's tensor-core kernel on host arrays
 * (its parity test): x is H x W pixels of cin channels (pixel-major,
 * channels innermost), w[n][9][cin] (tap = (dy+1)*3 + dx+1), bias[n] or
 * null; y[p][n] = act(bias + sum w x[p + dy W + dx]) in BF16 arithmetic with
 * FP32 accumulation, 0 outside the real_w x real_h corner; relu 0 or 1.
 * cin and n multiples of 16 (cin <= 128, n <= 256). */
int yz_conv3x3(int H, int W, int cin, int n, int real_w, int real_h, int relu, const float* x,
               const float* w, const float* bias, float* y);

/* ---------------------------------------------------------------------
 * Seam 3: the time step of the ConcZ model (a 2-D film with its
 * concentration resolved through the thickness on a zeta grid).  Replaces
 * _heightEq.TimeAdvance in ConcZ_Model_2D::Run (ConcZ_Model_2D.cpp:782):
 * CZ_HeightEquation_2D::TimeAdvance (CZ_HeightEquation_2D.cpp:1965-1974)
 * over C_SemiImplicitEquation::TimeAdvance / TimeStepTrial
 * (SemiImplicit.cpp:100-150) -- the semi-implicit film in two stages
 * (Solve, SolveStage: :1949-2020), its conservative update, the velocity
 * through the film (CalVelocity), the concentration equation on the moving
 * zeta grid (CZ_ConcEquation_2D.cpp) advanced by the same step, the
 * Aitken-relaxed coupling passes of the Marangoni film
 * (AfterTimeStepTrial, :207-386), RedistributeExcess / Deficit and the
 * LTE time-step control -- all on the device, both linear solves on this
 * library's SA-AMG BiCGStab.
 * ------------------------------------------------------------------- */
typedef struct yz_cz yz_cz;

typedef struct yz_cz_params
{
	int    nx, ny, nz;            /* grid sizes with the two ghost layers at each end (ny > 1) */
	int    bc[4];                 /* Xmin, Xmax, Ymin, Ymax: 0 Symmetry or 1 Periodic, in pairs (the
	                                 kinds the reference's CZ model implements:
	                                 CheckParameters.cpp:340-353 refuses the rest) */
	int    on_lap, on_sc, on_vg, on_hg, on_cf, on_evap;   /* Physics.* switches */
	int    ev_conc, ev_spatial, ev_hast;                 /* Raoult 0 / PowerN 1; uniform 0 / negPow 1; h* cap */
	int    dt_control, dt_keep_steps;                    /* Numerics.TimeStepControl */
	int    c_scheme;              /* Numerics.Convection.Concentration, YZ_SCHEME_* */
	yz_settings h_lin, c_lin;     /* the film's and the concentration's linear solver */
	double dx, dy, dzeta;         /* non-dimensional spacings; dzeta = 1 / (nz - 4) */
	double theta_h, theta_c;      /* Crank-Nicolson weights (0.5) */
	double dt, dt_old, dt_max, dt_min, time;
	double dt_change_factor, dt_criterion, dt_scale_floor;
	double As, Ma, Bo, Pgx, Pgy, Sp, Df, Ev;             /* non-dimensional numbers */
	double rot_center[2];
	double visc_c0, visc_base, visc_exp;  /* base * exp(exp (c - c0)), non-dimensional */
	double sig_c0, sig_base, sig_coef;    /* base + coef (c - c0) */
	double diff_c0, diff_base, diff_exp;
	double ev_mr, ev_ms, ev_pown, ev_concr, ev_negexp, ev_negrmax, ev_hast_h, ev_dr;
	double coupling_floor;        /* max(1e-10, 10 c_lin.epsilon) */
} yz_cz_params;

typedef struct yz_cz_stats
{
	int    steps;                 /* steps taken by this call */
	int    linear_iterations;     /* the film's BiCGStab iterations of the accepted trials (the
	                                 reference's BCGIterTotal) */
	int    conc_iterations;       /* the concentration's BiCGStab iterations, every solve */
	int    coupling_passes;       /* CouplingPasses() summed (CouplingPassTotal) */
	int    retries;               /* trials cut and repeated (dt control) */
	int    solves;                /* linear solves of either equation */
	double time, dt;              /* the clock and DT().now after the call */
	double device_ms;             /* the call on the model's stream (CUDA events) */
	long long launches;           /* kernels the call launched */
	/* the learned preconditioner of the film's solves (yz_cz_set_learned),
	 * for this call: film solves it converged, fallbacks to SA-AMG, its
	 * iterations, the training pairs held, the training's device time, the
	 * held-out error against the V-cycle and the last training loss (-1:
	 * not trained) */
	int    learned_solves, learned_fallbacks, learned_iterations, learned_samples;
	double learned_train_ms, learned_val_err, learned_loss;
} yz_cz_stats;

/* Build the model: the coordinates of the cell centres (xc, yc) and of the
 * faces below them (xf: the face between ix-1 and ix, yf likewise), and the
 * film h, substrate s (nx*ny, row jy*nx + ix) and concentration c (nx*ny*nz,
 * kz*nx*ny + jy*nx + ix) with their ghosts, as the reference's Build leaves
 * them; host arrays. */
int yz_cz_create(int device, const yz_cz_params* p, const double* xc, const double* xf, const double* yc,
                 const double* yf, const double* h, const double* s, const double* c, yz_cz** out);
int yz_cz_destroy(yz_cz* z);
/* nsteps time steps (TimeAdvance, then the clock's ++). */
int yz_cz_advance(yz_cz* z, int nsteps, yz_cz_stats* stats);
/* The film (nx*ny) and the concentration (nx*ny*nz) the model holds. */
int yz_cz_get_fields(yz_cz* z, double* h, double* c);
/* Replace them (host arrays; either may be null): the state the next step
 * starts from. */
int yz_cz_set_fields(yz_cz* z, const double* h, const double* c);
/* Preconditioner arithmetic (YZ_PREC_*) and AMG hierarchy reuse of both
 * equations' solves, from the next solve on (FP64, no reuse: the reference's). */
int yz_cz_set_precision(yz_cz* z, int precision);
int yz_cz_set_amg_reuse(yz_cz* z, int max_solves);
/* The FP32 V-cycle's launch shape of both equations' solves
 * (yz_solver_set_tuning). */
int yz_cz_set_tuning(yz_cz* z, int fuse_from, int coarse_lanes, int fine_sweeps);
/* The film's solves with a learned preconditioner of their own, as
 * yz_step_set_learned gives the well-mixed film's: the first collect_solves
 * SA-AMG film solves collect training pairs, the film solve after them
 * trains the network, and every later film solve tries it first within
 * cap_factor x the last SA-AMG solve's iterations.  The concentration's
 * solves keep SA-AMG.  Null: off. */
int yz_cz_set_learned(yz_cz* z, const yz_learned_cfg* cfg);
/* The pieces of one step on the present state, as the reference forms them
 * (its parity test): the film's assembly at the step's dt, its conservative
 * update with the film unchanged, the velocity and the concentration's
 * assembly with those fluxes.  Afterwards yz_cz_read copies a named array
 * ("h_A", "h_B", "h_colsrc", "h_qcapx", "h_qexpx", "h_qcapy", "h_qexpy",
 * "h_IA", "h_qx", "h_qy", "h_end", "h_dtdh", "ux", "uy", "c_A", "c_B",
 * "c_rhs", "c_react", "c_qx", "c_qy", "c_w") of up to cap values and
 * returns its length.  The model's state is not changed by the pieces. */
int yz_cz_parts(yz_cz* z);
long long yz_cz_read(yz_cz* z, const char* name, double* out, long long cap);
/* The patterns of the film's and the concentration's matrices in storage
 * order (the diagonal first), with the ghost-row flags; rowptr of n+1. */
int yz_cz_pattern(yz_cz* z, int which, int* rowptr, int* col, int* bc);
/* The same from the parameters alone (no device): which 0 the film, 1 the
 * concentration; returns the number of entries (arrays may be null to ask). */
int yz_cz_build_pattern(const yz_cz_params* p, int which, int* rowptr, int* col, int* bc);
/* The correctly rounded exp the ConcZ step's property laws use, on the
 * current device for n host values (its parity test against the host's). */
int yz_exp_cr(long long n, const double* x, double* y);

#ifdef __cplusplus
}
#endif

#endif
