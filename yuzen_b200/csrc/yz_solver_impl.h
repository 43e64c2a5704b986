// yz_solver_impl.h -- the device solver context behind yz_solver_* (C ABI).
#pragma once

#include "yz_common.cuh"
#include "../../include/yuzen_b200.h"

#include <memory>
#include <vector>

namespace yz {

class Learned;

//  Scalars of one BiCGStab run, in device memory (written by the block that
//  folds a reduction, read by the element-wise kernels and by the host).
struct Scal
{
	double normb, res, rho, rhoPrev, alpha, omega;
	double eps;              // tol * |b|
	int it, maxIter;         // iterations done, the cap
	int state;               // 0 running; see KState
	int bodies;              // iterations queued and run (the graph's loop count)
};

//  the state word of a BiCGStab run on the device
//  kTiny: |b| below twice the machine epsilon (x = 0, no iteration); kSkip:
//  the start residual already meets the tolerance, or no iteration allowed
enum KState { kRun = 0, kConv = 1, kConvHalf = 2, kBreak = 3, kNaN = 4, kCap = 5, kTiny = 6, kSkip = 7 };

//  TryBackoff, LinearSolverBackend.cpp:262-270
struct TryBackoff
{
	int skip = 0, wait = 16;
	bool Try() { if(skip > 0) { --skip; return false; } return true; }
	void Failed() { skip = wait; wait = (wait < 1024) ? 2 * wait : 1024; }
	void Converged() { wait = 16; }
};

struct Level
{
	int n = 0, nnz = 0;
	DBuf<int> ptr, col;
	DBuf<double> val;
	DBuf<double> M, f, x, t, xt;
	DBuf<int> agg;
	int nc = 0, pnnz = 0;
	DBuf<int> pptr, pcol, rptr, rcol;
	DBuf<double> pval, rval;
	bool direct = false;
	DBuf<double> inv;		// row-major dense inverse of the direct level
	//  the FP32 V-cycle (YZ_PREC_FP32_CYCLE): A (levels below the finest),
	//  SPAI0, P, R and the inverse rounded from the FP64 set-up, and the
	//  cycle's vectors
	DBuf<float> val32, M32, pval32, rval32, inv32, f32, x32, t32, xt32;
};

class Solver
{
public:
	//  stream null: the solver makes (and owns) a stream of its own;
	//  otherwise it runs on the caller's stream
	explicit Solver(int device, cudaStream_t stream = nullptr);
	~Solver();

	void SetPattern(int n, int nnz, const int *rowptr, const int *scol, const int *ssrc);
	int Solve(const yz_settings &set, const double *dValues, const double *dRhs, double *dX, int &iter, double &resid);
	int SolveHost(const yz_settings &set, const double *values, const double *rhs, double *x, int &iter, double &resid);

	std::vector<double> Memory() const;
	void SetMemory(const double *m, int len);
	int LevelCount() const;
	void LevelInfo(int l, int *rows, int *nnzA, int *nnzP, int *direct) const;
	void LevelCopy(int l, int *aptr, int *acol, double *aval, int *pptr, int *pcol, double *pval, int *agg);
	void Timing(double *setupMs, double *iterMs) const { if(setupMs) *setupMs = _setupMs; if(iterMs) *iterMs = _iterMs; }
	long long Launches() const { return _launches; }
	void SetPrecision(int precision);
	int Precision() const { return _precision; }
	void SetAmgReuse(int maxSolves);
	void SetGraphLoop(bool on) { _graphLoop = on; }
	void SetTuning(int fuseFrom, int coarseLanes, int fineSweeps);
	int Rebuilds() const { return _rebuilds; }
	//  the learned preconditioner (not owned): mode 0 off, 1 collect (the
	//  next `collectSolves` AMG solves feed the network's sample ring with up
	//  to `perSolve` (residual, V-cycle) pairs each), 2 use (the network in a
	//  flexible BiCGStab first, SA-AMG as the fallback)
	void SetLearned(Learned *L, int mode, int collectSolves, int perSolve, double capFactor);
	//  the film height for the network's features (a device vector of n; null: none)
	void SetAux(const double *dH) { _aux = dH; }
	int CollectLeft() const { return _collectLeft; }
	struct LearnedStats { int solves = 0, fallbacks = 0, iterations = 0, skipped = 0; };
	const LearnedStats &LStats() const { return _lstats; }
	int AmgIters() const { return _amgIters; }
	cudaStream_t Stream() const { return _st; }
	int Rows() const { return _n; }

private:
	enum { kPrecDiag = 0, kPrecAmg = 1, kPrecLearned = 2 };
	void BuildHierarchy(int coarseEnough);
	void DirectInverse(Level &L);
	void Cycle(size_t l, const double *f, double *x);
	Sten StenOf(size_t l) const;
	void RoundCycle();
	template<class TF, class TX> void Cycle32(size_t l, const TF *f, TX *x);
	int LanesFor(long long nnz, int n) const;
	bool CoarseCycleOn() const;
	static int CoarseBlocksPerSm();
	void LaunchCoarseCycle();
	void CoarsePreSmooth(int lanes, int n, const int *ptr, const int *col, const float *val, const float *M,
	                     const float *f, float *x, float *t);
	void CoarsePostSmooth(int lanes, int n, const int *ptr, const int *col, const float *val, const float *M,
	                      const float *f, const float *x, float *xout);
	void CoarseProlong(int lanes, int n, const int *pptr, const int *pcol, const float *pval, const float *xc,
	                   const float *x, float *xout);
	//  the first level whose way down and way up run fused (KDownFused,
	//  KUpFused); past the deepest level: none
	int FusedFrom() const;
	int FineSweeps() const;
	void CoarseDown(int lanes, int nc, const Level &L, const float *f, float *fc);
	void CoarseUp(int lanes, const Level &L, const float *f, const float *xc, float *x);
	const int *Halt() const { return &_sc.get()->state; }
	void ApplyPrec(int kind, const double *r, double *z);
	void EnqueueIteration(int kind);
	void RunIterations(int kind);
	//  the BiCGStab loop as a CUDA graph (a conditional while node whose body
	//  is one iteration); kept across solves while the hierarchy is reused
	struct LoopGraph
	{
		cudaGraph_t graph = nullptr;
		cudaGraphExec_t exec = nullptr;
		long long perBody = 0;
		unsigned long long key = ~0ull;       // the pattern/precision and hierarchy it was built for
	};
	void BuildLoopGraph(int kind, LoopGraph &g);
	static void FreeLoopGraph(LoopGraph &g);
	bool BiCGStab(int kind, int maxIter, double tol, int &itOut, double &errOut);
	double BreakdownResidual();
	int ReadInt(const int *d);
	void ReadScal();
	int ScanCounts(const int *cnt, int *out, int n, const int *flag = nullptr, int *flagOut = nullptr);
	int Gemm(int nx, const int *xptr, const int *xcol, const double *xval, const int *yptr, const int *ycol,
	         const double *yval, DBuf<int> &cptr, DBuf<int> &ccol, DBuf<double> &cval);
	RedScratch Red(int site);

	int _device;
	cudaStream_t _st = nullptr;
	bool _ownStream = true;
	cudaEvent_t _ev0 = nullptr, _ev1 = nullptr, _ev2 = nullptr;
	int _n = 0, _nnz = 0;
	std::vector<int> _hptr, _hcol;
	DBuf<int> _ssrc;
	DBuf<int> _sellOff, _sellCol;     // the finest level in SELL-32 (slice offsets, columns)
	DBuf<double> _sellVal;
	DBuf<float> _sellVal32;           // its FP32 copy, read by the FP32 V-cycle
	DBuf<unsigned char> _stenSlice;   // the slices whose rows are the stencil's
	Sten _sten = Sten();
	size_t _sellSize = 0;
	int _precision = YZ_PREC_FP64;
	DBuf<double> _values, _rhs, _xio;
	std::vector<std::unique_ptr<Level>> _levels;   // grows, never shrinks
	size_t _nlev = 0;                              // the levels of the present hierarchy
	bool _haveH = false;
	//  Krylov vectors
	DBuf<double> _b, _x, _x0, _r, _rh, _p, _v, _s, _ph, _sh, _t, _m;
	DBuf<double> _part;
	int _partBlocks = 1;
	DBuf<unsigned> _counters;
	DBuf<Scal> _sc;
	Scal *_hsc = nullptr;
	int *_hint = nullptr;      // pinned: totals and flags read back together
	Scal *_hring = nullptr;    // pinned: the state after the last two iterations
	cudaEvent_t _evRing[2] = {nullptr, nullptr};
	DBuf<int> _flags;
	//  set-up scratch
	DBuf<double> _dia;
	DBuf<unsigned char> _strong, _iso;
	DBuf<int> _icnt, _iptr, _icol, _ifill, _state, _flag, _rootId, _first, _cnt, _scan;
	DBuf<unsigned long long> _T0, _T1;
	DBuf<int> _gtCol;             // staged rows of a product (64 a row)
	DBuf<double> _gtVal;
	DBuf<int> _apPtr, _apCol;
	DBuf<double> _apVal;
	DBuf<double> _gj[2];          // [A | I] column-major, the panel multipliers
	DBuf<double> _gjPiv;
	DBuf<int> _gjRow;
	TryBackoff _offSpai;
	//  hierarchy reuse (0: a new set-up every solve, the reference's way)
	int _amgReuse = 0, _sinceBuild = 0, _freshIters = 0, _rebuilds = 0;
	bool _stale = false;
	int _hPrec = YZ_PREC_FP64;    // the precision the present hierarchy was set up in
	//  bumped whenever a pointer or size a loop graph holds may change: the
	//  pattern, precision or buffers (_epoch), the hierarchy (_epochH)
	unsigned _epoch = 0, _epochH = 0;
	//  launch shapes of the FP32 cycle's coarse levels (SetTuning): the first
	//  fused level (-1: YZ_FUSE_FROM or 2; 0: none) and the lanes a row (0:
	//  by the level's mean row length)
	int _fuseFrom = -1, _coarseLanes = 0, _fineSweeps = 0;
	LoopGraph _loop[3];
	bool _graphLoop = true;       // the loop as a CUDA graph (else from the stream)
	//  Solve's tail, queued behind a graph run: x into the caller's dX
	double *_tailDst = nullptr;
	const double *_tailSrc = nullptr;
	size_t _tailBytes = 0;
	bool _tailDone = false;
	//  the learned preconditioner
	Learned *_learned = nullptr;
	int _learnedMode = 0, _collectLeft = 0, _perSolve = 0, _collected = 0;
	bool _filmSolve = false;        // the present solve is one the network serves (a film's, SA-AMG)
	double _capFactor = 1.0;
	const double *_aux = nullptr;
	int _amgIters = 0;              // iterations of the last SA-AMG solve (the plain path's count)
	TryBackoff _offLearned;
	LearnedStats _lstats;
	DBuf<double> _zs;               // a collected pair's V-cycle output
	//  the persistent coarse cycle: its grid, barrier words and error word
	bool _coarseOn = true;
	int _coarseBlocks = 0;
	DBuf<unsigned> _coarseBar;
	DBuf<int> _coarseErr;
	double _setupMs = 0, _iterMs = 0;
	long long _launches = 0;
};

double DeviceDot(int n, const double *hx, const double *hy);
void DeviceSpmv(int n, int nnz, const int *rowptr, const int *col, const double *val, const double *hx, double *hy);
const char *LastError();
void TimeSelect(const char *name);
void DotNoAlloc(int n, const double *dx, const double *dy, double *dout, cudaStream_t st);
long long NoAllocMaxElements();
void TimeRead(double *ms, long long *count);
void FaultInject(long at, long count);

} // namespace yz
