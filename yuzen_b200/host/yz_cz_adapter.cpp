/*
 * yz_cz_adapter.cpp -- seam 3 on the reference's side: the time step of the
 * reference's ConcZ model handed to the device.
 *
 * The reference's step is _heightEq.TimeAdvance in ConcZ_Model_2D::Run
 * (ConcZ_Model_2D.cpp:782; CZ_HeightEquation_2D::TimeAdvance,
 * CZ_HeightEquation_2D.cpp:1965-1974) with the clock advance of the loop
 * (TimeSteps.cpp:121-160).  This file reads what that step needs out of the
 * reference's own objects -- the grids, the edges, the non-dimensional
 * groups, the property and evaporation laws, the linear-solver and time-step
 * settings (FillParams), the coordinates, the film, the substrate and the
 * concentration through the film (Gather) -- builds a yz_cz on the device,
 * advances it, and writes the film and the concentration back into the
 * model's fields (Scatter).
 *
 * The program built from it, yuzen_b200_cz (oracle/Makefile, target b200),
 * is the reference's driver with the CZ time loop on the device: it reads a
 * TOML case through C_Yuzen (ReadInputFile, Initialize: Yuzen.cpp:45,
 * 244-337) exactly as the reference does, runs Numerics.MaxSteps steps with
 * yz_cz_advance, puts the fields back into the reference's model and writes
 * them, read back from the model, with the step's counts and clock (a short
 * record described in main).
 *
 * The members read here are private in the reference; a maintainer adding
 * this code to the reference declares it a friend of the model classes.
 * Built here against the reference's headers unchanged, it opens their
 * access specifiers by macro, as the probe does.
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
#include "ConcZ_Model_2D.h"
#undef private
#undef protected

#include "yuzen_b200.h"

using namespace yuzen;

namespace {

//  every field of yz_cz_params from the object of the reference that holds it
void FillParams(ConcZ_Model_2D *m, yz_cz_params &p)
{
	std::memset(&p, 0, sizeof p);
	C_Grid3D *G3 = m->_field.GetGridPtr3();
	auto &he = m->_heightEq;
	auto &ce = m->_concEq;
	const BoundaryCondition2D &bc = m->_boundary;
	NonDimensionalNumbers &nd = m->_NonDim;
	p.nx = G3->nx(); p.ny = G3->ny(); p.nz = G3->nz();
	p.bc[0] = (int)bc._tXmin; p.bc[1] = (int)bc._tXmax; p.bc[2] = (int)bc._tYmin; p.bc[3] = (int)bc._tYmax;
	p.on_lap = he._sw_LaplacePressure ? 1 : 0; p.on_sc = he._sw_SolutoCapillarity ? 1 : 0;
	p.on_vg = he._sw_VerticalGravity ? 1 : 0; p.on_hg = he._sw_HorizontalGravity ? 1 : 0;
	p.on_cf = he._sw_Centrifugal ? 1 : 0; p.on_evap = nd._evap.Enabled() ? 1 : 0;
	p.ev_conc = (int)nd._evap._t_ConcFunc; p.ev_spatial = (int)nd._evap._t_SpatialFunc;
	p.ev_hast = nd._evap._sw_Hast_modify ? 1 : 0;
	p.dt_control = he._adjustTimeStep ? 1 : 0; p.dt_keep_steps = he._adjustTimeKeepSteps;
	p.c_scheme = (int)ce._scheme.Scheme();
	p.h_lin.precondition = (int)he._bcg._set.precondition; p.h_lin.scaling = he._bcg._set.scaling ? 1 : 0;
	p.h_lin.max_iteration = he._bcg._set.maxIteration; p.h_lin.epsilon = he._bcg._set.epsilon;
	p.h_lin.conc = he._bcg._set.conc ? 1 : 0;
	p.c_lin.precondition = (int)ce._bcg._set.precondition; p.c_lin.scaling = ce._bcg._set.scaling ? 1 : 0;
	p.c_lin.max_iteration = ce._bcg._set.maxIteration; p.c_lin.epsilon = ce._bcg._set.epsilon;
	p.c_lin.conc = ce._bcg._set.conc ? 1 : 0;
	p.dx = G3->dx(); p.dy = G3->dy(); p.dzeta = G3->dz();
	p.theta_h = he._theta; p.theta_c = ce._theta;
	p.dt = m->_timeStep.DT().now; p.dt_old = m->_timeStep.DT().old;
	p.dt_max = m->_timeStep.DT().range_max; p.dt_min = m->_timeStep.DT().range_min;
	p.time = m->_timeStep.NowTime();
	p.dt_change_factor = he._adjustTimeChangeFactor; p.dt_criterion = he._adjustTimeCriterion;
	p.dt_scale_floor = he._adjustTimeScaleFloor;
	p.As = nd.As(); p.Ma = nd.Ma(); p.Bo = nd.Bo(); p.Pgx = nd.Pgx(); p.Pgy = nd.Pgy(); p.Sp = nd.Sp();
	p.Df = nd.Df(); p.Ev = nd.Ev();
	p.rot_center[0] = he._rotCenter[0]; p.rot_center[1] = he._rotCenter[1];
	p.visc_c0 = nd._viscosity._baseConc; p.visc_base = nd._viscosity._baseValue; p.visc_exp = nd._viscosity._exponent;
	p.sig_c0 = nd._surface_tension._baseConc; p.sig_base = nd._surface_tension._baseValue;
	p.sig_coef = nd._surface_tension._coef;
	p.diff_c0 = nd._diffusivity._baseConc; p.diff_base = nd._diffusivity._baseValue;
	p.diff_exp = nd._diffusivity._exponent;
	p.ev_mr = nd._evap._M_resin; p.ev_ms = nd._evap._M_solvent; p.ev_pown = nd._evap._powerN;
	p.ev_concr = nd._evap._ConcR; p.ev_negexp = nd._evap._NegPowExponent; p.ev_negrmax = nd._evap._NegPowRmax;
	p.ev_hast_h = nd._evap._h_ast; p.ev_dr = std::min(nd._evap._G.dx(), nd._evap._G.dy());
	p.coupling_floor = he._couplingFloor;
}

//  the coordinates of the cell centres and of the faces below them
void Coords(ConcZ_Model_2D *m, std::vector<double> &xc, std::vector<double> &xf, std::vector<double> &yc,
            std::vector<double> &yf)
{
	C_Grid2D *G2 = m->_field.GetGridPtr2();
	const int nx = G2->nx(), ny = G2->ny();
	xc.resize((size_t)nx); xf.resize((size_t)nx); yc.resize((size_t)ny); yf.resize((size_t)ny);
	for(int i = 0; i < nx; ++i) { xc[(size_t)i] = G2->X(G2->At<Zface>(i, 0)); xf[(size_t)i] = G2->XOf<Yedge>(i, 0); }
	for(int j = 0; j < ny; ++j) { yc[(size_t)j] = G2->Y(G2->At<Zface>(0, j)); yf[(size_t)j] = G2->YOf<Xedge>(0, j); }
}

//  the model's fields in the device's order: h, s at jy nx + ix, c at
//  (kz ny + jy) nx + ix
void Gather(ConcZ_Model_2D *m, std::vector<double> &h, std::vector<double> &s, std::vector<double> &c)
{
	C_Grid2D *G2 = m->_field.GetGridPtr2();
	C_Grid3D *G3 = m->_field.GetGridPtr3();
	const int nx = G3->nx(), ny = G3->ny(), nz = G3->nz();
	h.assign((size_t)nx * ny, 0.0); s.assign((size_t)nx * ny, 0.0); c.assign((size_t)nx * ny * nz, 0.0);
	for(int jy = 0; jy < ny; ++jy)
		for(int ix = 0; ix < nx; ++ix)
		{
			h[(size_t)jy * nx + ix] = m->_field.HH(G2->At<Zface>(ix, jy));
			s[(size_t)jy * nx + ix] = m->_field.SS(G2->At<Zface>(ix, jy));
		}
	for(int kz = 0; kz < nz; ++kz)
		for(int jy = 0; jy < ny; ++jy)
			for(int ix = 0; ix < nx; ++ix)
				c[((size_t)kz * ny + jy) * nx + ix] = m->_field.CC(G3->At<Cell>(ix, jy, kz));
}

//  the device's film and concentration back into the model's fields
void Scatter(ConcZ_Model_2D *m, const std::vector<double> &h, const std::vector<double> &c)
{
	C_Grid2D *G2 = m->_field.GetGridPtr2();
	C_Grid3D *G3 = m->_field.GetGridPtr3();
	const int nx = G3->nx(), ny = G3->ny(), nz = G3->nz();
	for(int jy = 0; jy < ny; ++jy)
		for(int ix = 0; ix < nx; ++ix) m->_field.HH(G2->At<Zface>(ix, jy)) = h[(size_t)jy * nx + ix];
	for(int kz = 0; kz < nz; ++kz)
		for(int jy = 0; jy < ny; ++jy)
			for(int ix = 0; ix < nx; ++ix)
				m->_field.CC(G3->At<Cell>(ix, jy, kz)) = c[((size_t)kz * ny + jy) * nx + ix];
}

//  The prologue of ConcZ_Model_2D::Run (ConcZ_Model_2D.cpp:714-735)
void RunPrologue(ConcZ_Model_2D *m)
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
	m->BuildRestart();
}

} // namespace

int main(int argc, char **argv)
{
	if(argc < 3) { std::fprintf(stderr, "usage: yuzen_b200_cz case.toml out.bin [device]\n"); return 2; }
	const int device = argc > 3 ? std::atoi(argv[3]) : 0;
	C_Yuzen solver;
	if(!solver.ReadInputFile(argv[1])) return 1;
	if(!solver.Initialize()) return 1;
	ConcZ_Model_2D *m = dynamic_cast<ConcZ_Model_2D *>(solver._model);
	if(!m) { std::fprintf(stderr, "yuzen_b200_cz: the case does not build the ConcZ model\n"); return 3; }
	RunPrologue(m);
	yz_cz_params p;
	FillParams(m, p);
	std::vector<double> xc, xf, yc, yf, h, s, c;
	Coords(m, xc, xf, yc, yf);
	Gather(m, h, s, c);
	yz_cz *z = nullptr;
	if(yz_cz_create(device, &p, xc.data(), xf.data(), yc.data(), yf.data(), h.data(), s.data(), c.data(), &z) != 0)
	{
		std::fprintf(stderr, "yuzen_b200_cz: %s\n", yz_last_error());
		return 4;
	}
	const int steps = (int)m->_inputParam->Numerics.MaxSteps;
	yz_cz_stats stats;
	std::memset(&stats, 0, sizeof stats);
	auto t0 = std::chrono::steady_clock::now();
	const int ret = yz_cz_advance(z, steps, &stats);
	auto t1 = std::chrono::steady_clock::now();
	if(ret != 0)
	{
		std::fprintf(stderr, "yuzen_b200_cz: %s\n", yz_last_error());
		yz_cz_destroy(z);
		return 5;
	}
	yz_cz_get_fields(z, h.data(), c.data());
	Scatter(m, h, c);
	yz_cz_destroy(z);
	//  the state the run ends on, read back from the reference's own fields
	std::vector<double> h1, s1, c1;
	Gather(m, h1, s1, c1);
	FILE *f = std::fopen(argv[2], "wb");
	if(!f) return 6;
	//  a short record: magic, nx, ny, nz, steps, linear iterations, coupling
	//  passes, the clock, dt, the wall time, then h (nx*ny) and c (nx*ny*nz)
	std::fwrite("YZSEAM31", 1, 8, f);
	const int head[6] = {p.nx, p.ny, p.nz, stats.steps, stats.linear_iterations, stats.coupling_passes};
	std::fwrite(head, sizeof(int), 6, f);
	const double tail[3] = {stats.time, stats.dt, std::chrono::duration<double>(t1 - t0).count()};
	std::fwrite(tail, sizeof(double), 3, f);
	std::fwrite(h1.data(), sizeof(double), h1.size(), f);
	std::fwrite(c1.data(), sizeof(double), c1.size(), f);
	std::fclose(f);
	solver.Finalize();
	return 0;
}
