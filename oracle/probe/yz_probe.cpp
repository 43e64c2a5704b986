/*
 * yz_probe.cpp -- TEST INFRASTRUCTURE: the whole-step oracle.
 *
 * Builds a case through the reference's own driver (C_Yuzen::ReadInputFile,
 * Initialize: Yuzen.cpp:45,244-337), writes the state the implicit step starts
 * from, runs the reference's time loop (WellMixedModelBase.h:1235-1460) to
 * Numerics.MaxSteps, and writes the state it ends on.  Linked with the
 * reference library and the oracle linear-solver backend by oracle/Makefile.
 *
 *   yz_probe case.toml out.bin
 *
 * Layout of out.bin (little endian): magic "YZSTATE1"; int32 count of the
 * integer header, the integers; int32 count of the real header, the doubles;
 * then float64 arrays of nx*ny each (row = IL(ix,iy) = iy*nx + ix):
 * HH0, CC0, SS0 (after Build), HH1, CC1 (after the run); int32 rowptr[n+1],
 * col[nnz] of A's fixed pattern (storage order) and bc[n]; int32 n_c, nnz_c,
 * rowptr_c[n_c+1], col_c[nnz_c] of the concentration equation's pattern
 * (n_c = 0 without the WM concentration).
 * The header keys are listed in tests/golden/stateio.py.
 *
 * Private members are reached by compiling the reference headers with their
 * access specifiers opened; nothing of the reference is changed.
 */
#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>
#include <omp.h>

#define private public
#define protected public
#include "Yuzen.h"
#include "WellMixed_Model_2D.h"
#undef private
#undef protected

using namespace yuzen;

namespace {

typedef WellMixed_ModelBase<WM2D_Traits> Model2D;

void put(std::vector<int> &I, int v) { I.push_back(v); }
void put(std::vector<double> &D, double v) { D.push_back(v); }

void Fields(Model2D *m, std::vector<double> &h, std::vector<double> &c, std::vector<double> &s)
{
	C_Grid2D *G = m->_field.GetGridPtr();
	const int nx = G->nx(), ny = G->ny();
	h.assign((size_t)nx * ny, 0.0); c.assign((size_t)nx * ny, 0.0); s.assign((size_t)nx * ny, 0.0);
	for(int jy = 0; jy < ny; ++jy)
		for(int ix = 0; ix < nx; ++ix)
		{
			Zface z = G->At<Zface>(ix, jy);
			const size_t i = (size_t)G->IL(z);
			h[i] = m->_field.HH(z); c[i] = m->_field.CC(z); s[i] = m->_field.SS(z);
		}
}

} // namespace

int main(int argc, char **argv)
{
	if(argc != 3) { std::fprintf(stderr, "usage: yz_probe case.toml out.bin\n"); return 2; }
	C_Yuzen solver;
	if(!solver.ReadInputFile(argv[1])) return 1;
	if(!solver.Initialize()) return 1;
	Model2D *m = dynamic_cast<Model2D*>(solver._model);
	if(!m) { std::fprintf(stderr, "yz_probe: only the 2-D well-mixed model is probed\n"); return 3; }
	Input &inp = *m->_inputParam;
	NonDimensionalNumbers &nd = m->_NonDim;
	//  The prologue of WellMixed_ModelBase::Run (WellMixedModelBase.h:1235-1257),
	//  repeated by Run itself: the step capped by the output intervals, and a
	//  restart read (its ghosts set by the boundary conditions)
	{
		double max_dt = m->_timeStep.MaxDT(), val;
		const double T0 = nd.TimeScale();
		if(!inp.Output.FieldData.Listed()) { val = inp.Output.FieldData.TimeInterval / T0; if(val < max_dt) max_dt = val; }
		val = inp.Output.ProbeList.TimeInterval / T0;		if(val < max_dt) max_dt = val;
		val = inp.Output.GeneralHistory.TimeInterval / T0;	if(val < max_dt) max_dt = val;
		val = inp.Output.CalcInfo.TimeInterval / T0;		if(val < max_dt) max_dt = val;
		m->_timeStep.SetMaxDT(max_dt);
		if(m->_timeStep.MaxDT() < m->_timeStep.DT().initial) m->_timeStep.ChangeDT(m->_timeStep.MaxDT());
		if(inp.Restart.Enable) m->BuildRestart();
	}
	C_Grid2D *G = m->_field.GetGridPtr();
	auto &he = m->_heightEq;
	const BoundaryCondition2D &bc = m->_boundary;

	std::vector<int> I;
	std::vector<double> D;
	put(I, G->nx()); put(I, G->ny());
	put(I, (int)bc._tXmin); put(I, (int)bc._tXmax); put(I, (int)bc._tYmin); put(I, (int)bc._tYmax);
	put(I, he._LaplacePressure.Enabled()); put(I, he._VerticalGravity.Enabled());
	put(I, he._ParallelGravity.Enabled()); put(I, he._SolutoCapillarity.Enabled());
	put(I, he._Centrifugal.Enabled()); put(I, he._DisjoiningPressure.Enabled());
	put(I, nd._evap.Enabled() ? 1 : 0); put(I, he._swConcField ? 1 : 0); put(I, nd.Mob().Slip() ? 1 : 0);
	put(I, he._adjustTimeStep ? 1 : 0);
	put(I, (int)nd._evap._t_ConcFunc); put(I, (int)nd._evap._t_SpatialFunc); put(I, nd._evap._sw_Hast_modify ? 1 : 0);
	put(I, he._MaxIterNK); put(I, he._MinIterNK); put(I, he._jacobiInterval);
	put(I, (int)he._bcg._set.precondition); put(I, he._bcg._set.scaling ? 1 : 0); put(I, he._bcg._set.maxIteration);
	put(I, he._adjustTimeKeepSteps);
	put(I, (int)inp.Numerics.MaxSteps);
	put(I, he._Source.Enabled() ? 1 : 0);

	put(D, G->dx()); put(D, G->dy()); put(D, he._theta);
	put(D, m->_timeStep.DT().now); put(D, m->_timeStep.DT().range_max); put(D, m->_timeStep.DT().range_min);
	put(D, nd.As()); put(D, nd.Ma()); put(D, nd.Bo()); put(D, nd.Pgx()); put(D, nd.Pgy()); put(D, nd.Sp());
	put(D, nd.Dp()); put(D, nd.HStar()); put(D, nd.Pe()); put(D, nd.Mr()); put(D, nd.Df()); put(D, nd.Ev());
	put(D, nd.ExtentScale()); put(D, nd.HeightScale()); put(D, nd.TimeScale()); put(D, nd.Mob().Lambda());
	put(D, he._DisjoiningPressure._n); put(D, he._DisjoiningPressure._m); put(D, he._DisjoiningPressure._hstar);
	put(D, nd._viscosity._baseConc); put(D, nd._viscosity._baseValue); put(D, nd._viscosity._exponent);
	put(D, nd._surface_tension._baseConc); put(D, nd._surface_tension._baseValue); put(D, nd._surface_tension._coef);
	put(D, nd._diffusivity._baseConc); put(D, nd._diffusivity._baseValue); put(D, nd._diffusivity._exponent);
	put(D, nd._evap._M_resin); put(D, nd._evap._M_solvent); put(D, nd._evap._E0); put(D, nd._evap._powerN);
	put(D, nd._evap._NegPowExponent); put(D, nd._evap._NegPowRmax); put(D, nd._evap._ConcR); put(D, nd._evap._h_ast);
	put(D, he._EpsilonNK); put(D, he._EpsilonRelNK); put(D, he._bcg._set.epsilon);
	put(D, he._adjustTimeChangeFactor); put(D, he._adjustTimeCriterion); put(D, he._adjustTimeScaleFloor);
	put(D, G->X(G->At<Zface>(0, 0))); put(D, G->Y(G->At<Zface>(0, 0)));
	put(D, m->_timeStep.NowTime());
	//  the upwinded terms and the concentration equation
	{
		Zface z0 = G->At<Zface>(0, 0);
		const auto &ce = m->_concEq;
		put(I, (int)he._ParallelGravity._scheme.Scheme()); put(I, (int)ce._scheme.Scheme());
		put(I, ce._swConvection ? 1 : 0); put(I, ce._swDiffusion ? 1 : 0);
		put(I, (int)ce._bcg._set.precondition); put(I, ce._bcg._set.scaling ? 1 : 0); put(I, ce._bcg._set.maxIteration);
		put(I, ce._bcg._set.conc ? 1 : 0);
		put(D, G->X(G->HalfXm(z0))); put(D, G->Y(G->HalfYm(z0)));
		put(D, he._Centrifugal._Cnt[0]); put(D, he._Centrifugal._Cnt[1]);
		put(D, ce._bcg._set.epsilon); put(D, ce._theta);
		//  the nozzle (SourceBase)
		const auto &src = he._Source;
		put(I, src._numSubRegion); put(I, src._concSupplied ? 1 : 0);
		put(D, src._Radius); put(D, src._flowRate); put(D, src._timeConstant); put(D, src._armLength);
		put(D, src._armX); put(D, src._armY); put(D, src._rotationRate); put(D, src._startAngle);
		put(D, src._slopeTime); put(D, src._mainTime); put(D, m->_timeStep.StartTime()); put(D, src._Conc);
	}

	std::vector<double> h0, c0, s0;
	Fields(m, h0, c0, s0);
	const CRS_Matrix &A = he._crsA;
	const int n = A.RowSize(), nnz = A.NonZero();
	std::vector<int> rowptr(A.RowPtrData(), A.RowPtrData() + n + 1), col(A.ColIndData(), A.ColIndData() + nnz), flag(n);
	for(int i = 0; i < n; ++i) flag[(size_t)i] = A.IsBC(i) ? 1 : 0;
	//  the concentration equation's pattern (none without ConcField = WM)
	std::vector<int> crow, ccol;
	if(he._swConcField)
	{
		const CRS_Matrix &Ac = m->_concEq._crsA;
		crow.assign(Ac.RowPtrData(), Ac.RowPtrData() + Ac.RowSize() + 1);
		ccol.assign(Ac.ColIndData(), Ac.ColIndData() + Ac.NonZero());
	}

	//  the energy budget (WellMixed_ModelBase::EnergyEval) of the film the
	//  step starts from and of the one it ends on
	m->EnergyEval();
	const double enF0 = m->_enF, enD0 = m->_enD;
	auto t0 = std::chrono::steady_clock::now();
	m->Run();
	auto t1 = std::chrono::steady_clock::now();
	m->EnergyEval();
	const double enF1 = m->_enF, enD1 = m->_enD;
	solver.Finalize();
	std::vector<double> h1, c1, s1;
	Fields(m, h1, c1, s1);
	put(D, std::chrono::duration<double>(t1 - t0).count());
	put(D, m->_timeStep.NowTime());
	put(D, enF0); put(D, enD0); put(D, enF1); put(D, enD1);
	//  with Output.Energy, the energy dissipated over the run and the balance
	//  of its last step (WellMixedModelBase.h:1405-1411)
	put(D, m->_enDiss); put(D, m->_enBal);
	put(I, (int)m->_timeStep.TimeStep());
	put(I, m->Diverged() ? 1 : 0);

	FILE *f = std::fopen(argv[2], "wb");
	if(!f) return 4;
	std::fwrite("YZSTATE1", 1, 8, f);
	const int ni = (int)I.size(), nd_ = (int)D.size();
	std::fwrite(&ni, sizeof(int), 1, f); std::fwrite(I.data(), sizeof(int), I.size(), f);
	std::fwrite(&nd_, sizeof(int), 1, f); std::fwrite(D.data(), sizeof(double), D.size(), f);
	for(const std::vector<double> *v : {&h0, &c0, &s0, &h1, &c1}) std::fwrite(v->data(), sizeof(double), v->size(), f);
	std::fwrite(&n, sizeof(int), 1, f); std::fwrite(&nnz, sizeof(int), 1, f);
	std::fwrite(rowptr.data(), sizeof(int), rowptr.size(), f);
	std::fwrite(col.data(), sizeof(int), col.size(), f);
	std::fwrite(flag.data(), sizeof(int), flag.size(), f);
	const int cn = crow.empty() ? 0 : (int)crow.size() - 1, cnnz = (int)ccol.size();
	std::fwrite(&cn, sizeof(int), 1, f); std::fwrite(&cnnz, sizeof(int), 1, f);
	std::fwrite(crow.data(), sizeof(int), crow.size(), f);
	std::fwrite(ccol.data(), sizeof(int), ccol.size(), f);
	std::fclose(f);
	return 0;
}
