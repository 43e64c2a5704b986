/*
 * yz_step_adapter.cpp -- seam 2 on the reference's side: the implicit step of
 * a 2-D well-mixed model of the reference handed to the device.
 *
 * The reference's step is WellMixed_HeightEquation_2D::TimeAdvance
 * (C_NewtonKantorovich::TimeAdvance, NewtonKantorovich.cpp:424-486) with the
 * clock advance of the model loop (WellMixedModelBase.h:1334, TimeSteps.cpp:
 * 121-160).  This file reads what that step needs out of the reference's own
 * objects -- the grid, the boundary conditions, the non-dimensional groups,
 * the property and evaporation laws, the Newton, linear-solver and time-step
 * settings (FillParams), the film, concentration and substrate (Gather) --
 * builds a yz_step on the device, advances it, and writes the film and
 * concentration back into the model's fields (Scatter).
 *
 * The program built from it, yuzen_b200_step (oracle/Makefile, target b200),
 * is the reference's driver with the time loop on the device: it reads a
 * TOML case through C_Yuzen (ReadInputFile, Initialize: Yuzen.cpp:45,
 * 244-337) exactly as the reference does, runs Numerics.MaxSteps steps with
 * yz_step_advance, puts the fields back into the reference's model and writes
 * them, read back from the model, with the step's counts and clock (a short
 * record described in main), so that a test compares the device's run of a
 * case with the reference's.
 *
 * The members read here are private or protected in the reference; a
 * maintainer adding this code to the reference declares it a friend of the
 * model classes.  Built here against the reference's headers unchanged, it
 * opens their access specifiers by macro, as the probe does.
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

#include "yuzen_b200.h"

using namespace yuzen;

namespace {

typedef WellMixed_ModelBase<WM2D_Traits> Model2D;

//  the step's parameters from the reference's model: every field of
//  yz_step_params from the object of the reference that holds it
void FillParams(Model2D *m, yz_step_params &p)
{
	std::memset(&p, 0, sizeof p);
	C_Grid2D *G = m->_field.GetGridPtr();
	auto &he = m->_heightEq;
	const auto &ce = m->_concEq;
	const BoundaryCondition2D &bc = m->_boundary;
	NonDimensionalNumbers &nd = m->_NonDim;
	Zface z0 = G->At<Zface>(0, 0);
	p.nx = G->nx(); p.ny = G->ny();
	p.bc[0] = (int)bc._tXmin; p.bc[1] = (int)bc._tXmax; p.bc[2] = (int)bc._tYmin; p.bc[3] = (int)bc._tYmax;
	p.dx = G->dx(); p.dy = G->dy();
	p.xmin = G->X(G->HalfXm(z0)); p.ymin = G->Y(G->HalfYm(z0));
	p.theta = he._theta;
	p.on_laplace = he._LaplacePressure.Enabled(); p.on_vgrav = he._VerticalGravity.Enabled();
	p.on_pgrav = he._ParallelGravity.Enabled(); p.on_marangoni = he._SolutoCapillarity.Enabled();
	p.on_centrifugal = he._Centrifugal.Enabled(); p.on_disjoining = he._DisjoiningPressure.Enabled();
	p.on_evap = nd._evap.Enabled() ? 1 : 0;
	p.conc_field = he._swConcField ? 1 : 0;
	p.Bo = nd.Bo(); p.Dp = nd.Dp(); p.hstar = he._DisjoiningPressure._hstar;
	p.disj_n = he._DisjoiningPressure._n; p.disj_m = he._DisjoiningPressure._m;
	p.lambda_slip = nd.Mob().Lambda(); p.Ev = nd.Ev();
	p.visc_c0 = nd._viscosity._baseConc; p.visc_base = nd._viscosity._baseValue; p.visc_exp = nd._viscosity._exponent;
	p.sig_c0 = nd._surface_tension._baseConc; p.sig_base = nd._surface_tension._baseValue;
	p.sig_coef = nd._surface_tension._coef;
	p.ev_conc_func = (int)nd._evap._t_ConcFunc; p.ev_spatial = (int)nd._evap._t_SpatialFunc;
	p.ev_hast_modify = nd._evap._sw_Hast_modify ? 1 : 0;
	p.ev_m_resin = nd._evap._M_resin; p.ev_m_solvent = nd._evap._M_solvent; p.ev_power_n = nd._evap._powerN;
	p.ev_conc_r = nd._evap._ConcR; p.ev_negpow_exp = nd._evap._NegPowExponent;
	p.ev_negpow_rmax = nd._evap._NegPowRmax; p.ev_h_ast = nd._evap._h_ast;
	p.nk_max = he._MaxIterNK; p.nk_min = he._MinIterNK; p.nk_eps = he._EpsilonNK; p.nk_eps_rel = he._EpsilonRelNK;
	p.lin.precondition = (int)he._bcg._set.precondition; p.lin.scaling = he._bcg._set.scaling ? 1 : 0;
	p.lin.max_iteration = he._bcg._set.maxIteration; p.lin.epsilon = he._bcg._set.epsilon; p.lin.conc = 0;
	p.dt_control = he._adjustTimeStep ? 1 : 0; p.dt_keep_steps = he._adjustTimeKeepSteps;
	p.dt = m->_timeStep.DT().now; p.dt_max = m->_timeStep.DT().range_max; p.dt_min = m->_timeStep.DT().range_min;
	p.dt_change_factor = he._adjustTimeChangeFactor; p.dt_criterion = he._adjustTimeCriterion;
	p.dt_scale_floor = he._adjustTimeScaleFloor;
	p.t_start = m->_timeStep.NowTime();
	p.conv_height = (int)he._ParallelGravity._scheme.Scheme();
	p.Pgx = nd.Pgx(); p.Pgy = nd.Pgy(); p.Sp = nd.Sp();
	p.rot_x = he._Centrifugal._Cnt[0]; p.rot_y = he._Centrifugal._Cnt[1];
	p.As = nd.As(); p.Ma = nd.Ma();
	p.conv_conc = (int)ce._scheme.Scheme();
	p.conc_convection = ce._swConvection ? 1 : 0; p.conc_diffusion = ce._swDiffusion ? 1 : 0;
	p.theta_c = ce._theta;
	p.Df = nd.Df(); p.diff_c0 = nd._diffusivity._baseConc; p.diff_base = nd._diffusivity._baseValue;
	p.diff_exp = nd._diffusivity._exponent;
	p.lin_conc.precondition = (int)ce._bcg._set.precondition; p.lin_conc.scaling = ce._bcg._set.scaling ? 1 : 0;
	p.lin_conc.max_iteration = ce._bcg._set.maxIteration; p.lin_conc.epsilon = ce._bcg._set.epsilon;
	p.lin_conc.conc = ce._bcg._set.conc ? 1 : 0;
	//  the nozzle (SourceBase.cpp:20-38)
	const auto &src = he._Source;
	p.on_source = src.Enabled() ? 1 : 0;
	p.src_subregions = src._numSubRegion;
	p.src_radius = src._Radius; p.src_rate = src._flowRate; p.src_tau = src._timeConstant;
	p.src_arm = src._armLength; p.src_arm_x = src._armX; p.src_arm_y = src._armY;
	p.src_omega = src._rotationRate; p.src_angle0 = src._startAngle;
	p.src_ramp = src._slopeTime; p.src_plateau = src._mainTime; p.src_t0 = m->_timeStep.StartTime();
	p.src_supplied = src._concSupplied ? 1 : 0; p.src_conc = src._Conc;
}

//  the model's fields in the device's row order IL(ix, iy) = iy nx + ix
void Gather(Model2D *m, std::vector<double> &h, std::vector<double> &c, std::vector<double> &s)
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

//  the device's film and concentration back into the model's fields
void Scatter(Model2D *m, const std::vector<double> &h, const std::vector<double> &c)
{
	C_Grid2D *G = m->_field.GetGridPtr();
	const int nx = G->nx(), ny = G->ny();
	for(int jy = 0; jy < ny; ++jy)
		for(int ix = 0; ix < nx; ++ix)
		{
			Zface z = G->At<Zface>(ix, jy);
			const size_t i = (size_t)G->IL(z);
			m->_field.HH(z) = h[i];
			m->_field.CC(z) = c[i];
		}
}

//  The prologue of WellMixed_ModelBase::Run (WellMixedModelBase.h:1235-1257):
//  the step capped by the output intervals, and a restart read
void RunPrologue(Model2D *m)
{
	Input &inp = *m->_inputParam;
	const double T0 = m->_NonDim.TimeScale();
	double max_dt = m->_timeStep.MaxDT(), val;
	if(!inp.Output.FieldData.Listed()) { val = inp.Output.FieldData.TimeInterval / T0; if(val < max_dt) max_dt = val; }
	val = inp.Output.ProbeList.TimeInterval / T0;		if(val < max_dt) max_dt = val;
	val = inp.Output.GeneralHistory.TimeInterval / T0;	if(val < max_dt) max_dt = val;
	val = inp.Output.CalcInfo.TimeInterval / T0;		if(val < max_dt) max_dt = val;
	m->_timeStep.SetMaxDT(max_dt);
	if(m->_timeStep.MaxDT() < m->_timeStep.DT().initial) m->_timeStep.ChangeDT(m->_timeStep.MaxDT());
	if(inp.Restart.Enable) m->BuildRestart();
}

} // namespace

int main(int argc, char **argv)
{
	if(argc < 3) { std::fprintf(stderr, "usage: yuzen_b200_step case.toml out.bin [device]\n"); return 2; }
	const int device = argc > 3 ? std::atoi(argv[3]) : 0;
	C_Yuzen solver;
	if(!solver.ReadInputFile(argv[1])) return 1;
	if(!solver.Initialize()) return 1;
	Model2D *m = dynamic_cast<Model2D *>(solver._model);
	if(!m) { std::fprintf(stderr, "yuzen_b200_step: the device step takes the 2-D well-mixed model\n"); return 3; }
	RunPrologue(m);
	yz_step_params p;
	FillParams(m, p);
	std::vector<double> h, c, s;
	Gather(m, h, c, s);
	yz_step *st = nullptr;
	if(yz_step_create(device, &p, h.data(), c.data(), s.data(), &st) != 0)
	{
		std::fprintf(stderr, "yuzen_b200_step: %s\n", yz_last_error());
		return 4;
	}
	const int steps = (int)m->_inputParam->Numerics.MaxSteps;
	yz_step_stats stats;
	std::memset(&stats, 0, sizeof stats);
	auto t0 = std::chrono::steady_clock::now();
	const int ret = yz_step_advance(st, steps, &stats);
	auto t1 = std::chrono::steady_clock::now();
	if(ret != 0)
	{
		std::fprintf(stderr, "yuzen_b200_step: %s\n", yz_last_error());
		yz_step_destroy(st);
		return 5;
	}
	yz_step_get_fields(st, h.data(), c.data());
	Scatter(m, h, c);
	yz_step_destroy(st);
	//  the state the run ends on, read back from the reference's own fields
	std::vector<double> h1, c1, s1;
	Gather(m, h1, c1, s1);
	FILE *f = std::fopen(argv[2], "wb");
	if(!f) return 6;
	//  a short record: magic, steps, Newton passes, linear iterations, the
	//  clock, the wall time, then h and c (nx*ny each, IL order)
	std::fwrite("YZSEAM21", 1, 8, f);
	const int head[4] = {p.nx, p.ny, stats.steps, stats.newton_iterations};
	std::fwrite(head, sizeof(int), 4, f);
	const double tail[3] = {stats.time, std::chrono::duration<double>(t1 - t0).count(), (double)stats.linear_iterations};
	std::fwrite(tail, sizeof(double), 3, f);
	std::fwrite(h1.data(), sizeof(double), h1.size(), f);
	std::fwrite(c1.data(), sizeof(double), c1.size(), f);
	std::fclose(f);
	solver.Finalize();
	return 0;
}
