// yz_step_impl.h -- the device step context behind yz_step_* (C ABI).
#pragma once

#include "yz_bc.h"

#include "yz_learned.h"
#include "yz_physics.cuh"
#include "yz_solver_impl.h"

#include <memory>
#include <vector>

namespace yz {
namespace phys {
struct ConcIn;
} // namespace phys
} // namespace yz

namespace yz {

void BuildPattern2D(const yz_step_params &p, std::vector<int> &rowptr, std::vector<int> &col,
                    std::vector<int> &isbc, std::vector<int> &ghost, std::vector<int> &partner,
                    BcPlan *plan = nullptr);
void CheckParams(const yz_step_params &p);

//  a SatisfyBCRows plan (yz_bc.h) on the device
struct DevBcPlan
{
	int nSets = 0;
	bool simple = true;
	DBuf<int> m, rowOff, matOff, row, termOff, termCol, piv;
	DBuf<double> rhs, termVal, fac, U;
	void Upload(const BcPlan &P, cudaStream_t st)
	{
		nSets = (int)P.setM.size();
		simple = P.simple;
		if(simple) return;
		m.upload(P.setM.data(), P.setM.size(), st);
		rowOff.upload(P.setRowOff.data(), P.setRowOff.size(), st);
		matOff.upload(P.setMatOff.data(), P.setMatOff.size(), st);
		row.upload(P.row.data(), P.row.size(), st);
		rhs.upload(P.rowRhs.data(), P.rowRhs.size(), st);
		termOff.upload(P.termOff.data(), P.termOff.size(), st);
		termCol.upload(P.termCol.data(), P.termCol.size(), st);
		termVal.upload(P.termVal.data(), P.termVal.size(), st);
		piv.upload(P.piv.data(), P.piv.size(), st);
		fac.upload(P.fac.data(), P.fac.size(), st);
		U.upload(P.U.data(), P.U.size(), st);
	}
	BcSets Sets(const double *rhsVec) const
	{
		BcSets S;
		S.n = nSets;
		S.m = m.get(); S.rowOff = rowOff.get(); S.matOff = matOff.get(); S.row = row.get();
		S.termOff = termOff.get(); S.termCol = termCol.get(); S.piv = piv.get();
		S.rhs = rhs.get(); S.termVal = termVal.get(); S.fac = fac.get(); S.U = U.get();
		S.rhsVec = rhsVec;
		return S;
	}
};

class Step
{
public:
	Step(int device, const yz_step_params &p, const double *h, const double *c, const double *s);
	~Step();
	void Advance(int nsteps, yz_step_stats &stats);
	void GetFields(double *h, double *c);
	void Energy(double &F, double &D);
	void SetEnergy(bool on);
	void SetFields(const double *h, const double *c);
	//  the whole state a later step depends on, as a flat array of doubles
	size_t StateSize() const;
	void GetState(double *out);
	void SetState(const double *in, size_t len);
	int Pattern(int *rowptr, int *col, int *bc) const;
	void System(const double *hOld, const double *h, double dt, double *ia, double *rhs);
	int ConcPattern(int *rowptr, int *col) const;
	void ConcSystem(const double *h, const double *c, double dt, double *val, double *rhs);
	long long Launches() const { return _solver->Launches(); }
	void SetPrecision(int precision)
	{
		_solver->SetPrecision(precision);
		if(_solverC) _solverC->SetPrecision(precision);
		_precision = precision;
	}
	void SetGraphLoop(bool on)
	{
		_solver->SetGraphLoop(on);
		if(_solverC) _solverC->SetGraphLoop(on);
		_graphLoop = on;
	}
	void SetTuning(int fuseFrom, int coarseLanes, int fineSweeps)
	{
		_solver->SetTuning(fuseFrom, coarseLanes, fineSweeps);
		if(_solverC) _solverC->SetTuning(fuseFrom, coarseLanes, fineSweeps);
	}
	void SetAmgReuse(int maxSolves)
	{
		_solver->SetAmgReuse(maxSolves);
		if(_solverC) _solverC->SetAmgReuse(maxSolves);
		_amgReuse = maxSolves;
	}
	int Rows() const { return _n; }
	int Nnz() const { return _nnz; }
	//  the learned preconditioner of the film's solves (null: off)
	void SetLearned(const yz_learned_cfg *cfg);
	Learned *GetLearned() const { return _learned.get(); }

private:
	enum { kSlotRhs = 0, kSlotDelta = 1, kSlotPhi = 2, kSlotMove = 3, kSlotLte = 4, kSlotBad = 5, kSlotCorr = 6,
	       kSlotFlags = 7 };
	void BuildPattern();
	void BuildCoef();
	void FaceProps(const double *H, const double *C, bool J);
	void SatisfyGhosts(double *x);
	//  the concentration's ghost rows of x exactly, with the right-hand side
	//  rhsVec (a vector over the rows) or the equation's own (null)
	void SatisfyConcGhosts(double *x, const double *rhsVec);
	void ConcUpdate(int mode, double dt);
	void ConcInputs(phys::ConcIn &in) const;
	void UpdateSource(double dt);
	void Assemble(int mode, const double *hField, const double *cField, double dt);
	bool NKLoop(int &iter, double &resid, yz_step_stats &stats);
	//  the concentration equation
	void BuildConc(const double *cHost);
	int FaceFluxes(const double *H, const double *C, double *Fx, double *Fy, double dt, bool withEvap);
	void ConcAssemble(double dt);
	int ConcSolve(yz_step_stats &stats);
	bool ConcPass(double dt, yz_step_stats &stats);
	void ConcCommit(double dt, yz_step_stats &stats);
	void Redistribute();
	void MoveExcess(bool lower);
	RedScratch StepRed(int site);
	double ReadMax(int slot);
	void ZeroMax(int slot);

	int _device;
	yz_step_params _p;
	phys::Coef _k;
	std::unique_ptr<Solver> _solver;
	cudaStream_t _st = nullptr;
	cudaEvent_t _e0 = nullptr, _e1 = nullptr, _eA = nullptr, _eB = nullptr;
	int _n = 0, _nnz = 0;
	std::vector<int> _rowptr, _col, _isbc, _ghost, _partner;
	DBuf<int> _dRowptr, _dGhost, _dPartner;
	DBuf<unsigned char> _dIsbc;
	//  the ghost rows (yz_bc.h): the Newton matrix's values on them and their
	//  right-hand side, and the SatisfyBCRows programme (used unless every
	//  ghost row copies one cell)
	BcPlan _bc;
	DBuf<int> _dBcPos;
	DBuf<double> _dBcVal, _dBcRhs;
	int _nBcVal = 0;
	DevBcPlan _dBc;
	//  the concentration equation's ghost rows (its own plan; b: their
	//  right-hand side, from the start concentration)
	BcPlan _bcC;
	DevBcPlan _dBcC;
	DBuf<double> _dBcCRhs;
	DBuf<int> _dColC;
	DBuf<double> _cPre, _G2x, _G2y;          // Reconstruct: c1 as solved, the faces' solute fluxes
	DBuf<double> _src;                       // the nozzle's supply of the step (Physics.Source)
	//  fields: the committed film h (field), c, s; phi_old, phi_old2, phi_new,
	//  phi_guess; A h at phi_old and at the guess; the system
	DBuf<double> _h, _c, _s, _hOld, _hOld2, _hNew, _guess, _axOld, _axGuess, _rhs, _delta, _evapOld, _evapB, _ia;
	DBuf<unsigned long long> _red;
	DBuf<double> _faceMem;
	DBuf<double> _enFx, _enFy, _enOut;       // the energy budget's face fluxes and its two sums
	DBuf<double> _upMem;                     // the limited upwind terms' faces (UpBuf)
	//  the energy history (Output.Energy)
	bool _energyOn = false;
	double _enF = 0, _enD = 0, _enDiss = 0, _enBal = 0;
	phys::FaceBuf _fb;
	//  the concentration equation: its pattern and solver; c0 (its phi_old),
	//  the working field's c, the limiter state, the c of the last pass,
	//  the solution c1 and the one before the solves that complete the step,
	//  the correction d (and the next solve's guess), its system; the face
	//  volume fluxes at the start of the step (F0) and at the pass's film (F1),
	//  the evaporation of the step, ConsistentFluxes' and MoveExcess' scratch
	bool _conc = false;
	phys::ConcCoef _kc;
	std::unique_ptr<Solver> _solverC;
	int _precision = YZ_PREC_FP64, _amgReuse = 0;
	bool _graphLoop = true;
	int _nnzC = 0;
	std::vector<int> _rowptrC, _colC;
	DBuf<int> _dRowptrC, _dPartnerAll;
	DBuf<double> _cw, _c0, _cLim, _cPrev, _cx, _cxLast, _dC, _rhsC, _iaC, _F0x, _F0y, _F1x, _F1y, _evpStep;
	DBuf<double> _rho, _rowSum, _accY, _room, _give, _sums, _partStep;
	DBuf<unsigned int> _cntStep;
	DBuf<int> _iflags;
	double _coupled = 0;
	//  the clock (C_TimeSteps) and the Newton state
	double _dt = 0, _dtOld = 0, _time = 0, _pendingDt = 0;
	int _adjustCount = 0, _nkIter = 0;
	double _ewEta = 0, _ewRhsPrev = 0, _extrapMove = 0, _lastResid = 0;
	bool _extrapBlocked = false;
	//  the learned preconditioner: the network (its weights and sample
	//  ring), its settings and what its training reported
	std::unique_ptr<Learned> _learned;
	yz_learned_cfg _lcfg{};
	double _lValErr = -1.0, _lLoss = -1.0;
	void TrainLearned(yz_step_stats &stats);
};

} // namespace yz
