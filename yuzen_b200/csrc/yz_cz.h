// yz_cz.h -- the ConcZ model's time step on the device (yz_cz_* of the C
// ABI): the film height h (nx x ny, row IL(ix, jy) = jy nx + ix) and the
// concentration c resolved through the film on a zeta grid (nx x ny x nz,
// IL(ix, jy, kz) = kz nx ny + jy nx + ix), both with two ghost layers at each
// end of every axis.
//
// The step follows CZ_HeightEquation_2D (model/ConcZ/CZ2D/
// CZ_HeightEquation_2D.cpp) and CZ_ConcEquation_2D (CZ_ConcEquation_2D.cpp)
// over C_SemiImplicitEquation (numerics/SemiImplicit.cpp):
//
//   TimeAdvance        phi_old2 <- phi_old <- phi_new, then trials until the
//                      LTE test (ImplicitSolver.cpp:271-307) accepts one
//     Solve            SolveStage with the coefficients of the start of the
//                      step, then again with every coefficient at the
//                      midpoint (h halfway, c extrapolated)
//     SolveStage       SetMatrixA (the conservative film: face mobilities,
//                      the capillary term in the matrix, the rest on the
//                      right), A phi_old, I + theta dt A, the right-hand
//                      side, one BiCGStab solve
//     AfterTimeStepTrial  the conservative update through the face fluxes,
//                      dh/dt, the velocity through the film, the
//                      concentration step (two stages, or one per coupling
//                      pass with the Marangoni term: Aitken-relaxed passes
//                      until the midpoint settles), RedistributeExcess /
//                      Deficit, the ghosts of the end state
//
// Each loop of the reference over cells, faces or columns is one kernel here
// (one thread per row, face or column, the z loop inside the thread), with
// the reference's arithmetic in the reference's order; the sums over the
// film (the Aitken weights, the solute correction alpha) are fixed-order
// tree reductions.  Both equations solve on the library's SA-AMG BiCGStab
// (yz_solver), which restates the reference's backend.
#pragma once

#include "yuzen_b200.h"
#include "yz_common.cuh"
#include "yz_physics.cuh"
#include "yz_solver_impl.h"
#include "yz_learned.h"

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace yz {

//  the correctly rounded exp (yz_exp.h) of n host values on the current device
void ExpCrHost(long long n, const double *x, double *y);

//  the parameters this path takes (UsageError otherwise)
void CheckCzParams(const yz_cz_params &p);

void BuildCzPatterns(const yz_cz_params &p, std::vector<int> &rowptrH, std::vector<int> &colH, std::vector<int> &bcH,
                     std::vector<int> &rowptrC, std::vector<int> &colC, std::vector<int> &bcC);

//  what the kernels need, by value
struct CzCoef
{
	int nx, ny, nz;
	int perX, perY;          // both ends periodic (the ghost rows)
	int perXv, perYv;        // the minimum end periodic (the velocity's ghosts)
	int wall[4];             // BoundaryCondition::IsWall of Xmin, Xmax, Ymin, Ymax
	int onL, onSC, onVG, onHG, onCF, onEvap;
	double dx, dy, dzeta;
	double rdx, rdx2, rdx4, rdy, rdy2, rdy4, rdx2dy2, dx3, dy3;
	double As, Ma, Bo, Pgx, Pgy, Sp, Df, Ev, rot0, rot1;
	double diffC0, diffBase, diffExp;
	phys::Coef ev;           // the property laws and the evaporation (yz_physics.cuh)
	phys::Interp cI;         // Numerics.Convection.Concentration
	const double *xc, *xf, *yc, *yf;
};

class CzStep
{
public:
	CzStep(int device, const yz_cz_params &p, const double *xc, const double *xf, const double *yc, const double *yf,
	       const double *h, const double *s, const double *c);
	~CzStep();
	void Advance(int nsteps, yz_cz_stats &stats);
	void GetFields(double *h, double *c);
	void SetFields(const double *h, const double *c);
	void SetPrecision(int precision);
	void SetAmgReuse(int maxSolves);
	void SetTuning(int fuseFrom, int coarseLanes, int fineSweeps);
	void SetLearned(const yz_learned_cfg *cfg);
	void Parts();
	long long Read(const std::string &name, double *out, long long cap);
	int Pattern(int which, int *rowptr, int *col, int *bc) const;
	long long Launches() const { return _launches; }

private:
	//  the field the reference's kernels read (Field_CZ) and its copy at the
	//  start of the step (_field_tmp)
	void SetMatrixAH(const double *fH, const double *fC, double dt);
	void SolveStageH(const double *fH, const double *fC, double dt, int &iter, double &resid, int &ch);
	void SolveH(double dt, int &iter, double &resid, int &ch);
	void ConservativeUpdate(double dt);
	void CopyGhostsH(double *h);
	void CalDtDh(double dt);
	void CalVelocity(const double *fH, const double *fC);
	void BuildVolumeFluxes(const double *fH);
	void SetMatrixAC(const double *fH, const double *fC, double dt);
	void SetBcC(const double *fH, const double *fC, bool atEnd, double dt);
	void ApplyBoundaryRowsC(double *x);
	void ExplicitPartC(const double *x, double *Ax);
	int SolveStageC(const double *fH, const double *fC, double dt, int &iter, double &resid);
	int SolveC(const double *fH, double dt, int &iter, double &resid);
	int SolveAtMidpointC(const double *fH, const double *cmid, double dt, int &iter, double &resid);
	int SettleLimiterC(const double *fH, double dt, int &iter, double &resid);
	bool AfterTrial(double dt, yz_cz_stats &stats);
	void TrainLearned();
	void RedistributeExcess();
	void RedistributeDeficit();
	double Lte(double dt);

	double AbsMax(const double *x, long long n);
	bool Flag();
	void ZeroFlag();
	void Copy(double *dst, const double *src, size_t n);

	int _device;
	cudaStream_t _st = nullptr;
	yz_cz_params _p;
	CzCoef _k;
	int _n2, _n3, _nnzH, _nnzC;
	std::vector<int> _rowptrH, _colH, _bcH, _rowptrC, _colC, _bcC;
	std::unique_ptr<Solver> _solverH, _solverC;
	long long _launches = 0;
	//  the learned preconditioner of the film's solves
	std::unique_ptr<Learned> _learned;
	yz_learned_cfg _lcfg = {};
	double _lValErr = -1.0, _lLoss = -1.0, _lTrainMs = 0.0;

	DBuf<double> _xc, _xf, _yc, _yf;
	DBuf<int> _dRowptrH, _dColH, _dRowptrC, _dColC;
	DBuf<unsigned char> _dBcH, _dBcC;
	//  the field and its copy at the start of the step
	DBuf<double> _s, _fH, _fC, _tH, _tC;
	//  the film's equation
	DBuf<double> _hOld2, _hOld, _hNew, _A, _IA, _B, _Ax, _rhs, _colSrc, _dtdh, _hc, _hMid;
	DBuf<double> _D[2], _sig[2], _M[2], _qCap[2], _qExp[2], _q[2];
	//  the concentration's equation
	DBuf<double> _cOld2, _cOld, _cNew, _Ac, _IAc, _Bc, _Rc, _react, _Axc, _rhsc, _d, _ct, _Qx, _Qy, _W, _Ux, _Uy;
	DBuf<double> _kOld2, _kOld, _kNew;           // KeepStepStart
	DBuf<double> _ccPrev, _ccPrevKeep, _c0, _cm, _r, _rPrev, _mid, _prev;
	DBuf<double> _red;                           // reduction partials and results
	DBuf<unsigned long long> _max;
	DBuf<int> _flag;
	double _dt, _dtOld, _time, _pendingDt = 0;
	double _dtPrev = 1.0;
	bool _ccPrevSet = false;
	int _adjustCount = 0;
	int _couplingPasses = 0;
	long long _solves = 0, _concIters = 0;
	std::map<std::string, std::vector<double>> _parts;
};

} // namespace yz
