/*
 * yz_probe_cz.cpp -- TEST INFRASTRUCTURE: the oracle of the ConcZ model.
 *
 * Builds a case through the reference's own driver (C_Yuzen::ReadInputFile,
 * Initialize: Yuzen.cpp:45,244-337) with Physics.ConcField.Model = "CZ",
 * repeats the prologue of ConcZ_Model_2D::Run (ConcZ_Model_2D.cpp:714-735:
 * the step capped by the output intervals) and writes what the device step
 * starts from: the parameters, the film h and the substrate s (Nx x Ny, row
 * IL(ix, jy) = jy Nx + ix), the concentration c (Nx x Ny x Nz, IL(ix, jy, kz)
 * = kz Nx Ny + jy Nx + ix), the patterns of the film's and the
 * concentration's matrices (storage order) and their ghost-row flags.  Then
 *
 *   yz_probe_cz case.toml out.bin          runs the reference's time loop
 *                                          (ConcZ_Model_2D::Run) to
 *                                          Numerics.MaxSteps and writes the
 *                                          state it ends on;
 *   yz_probe_cz case.toml out.bin ... init=h.bin
 *                                          first replaces the film the case
 *                                          built by the nx*ny doubles of
 *                                          h.bin (row jy nx + ix, ghosts
 *                                          included): the field, its copy at
 *                                          the start of the step and the
 *                                          height equation's unknowns;
 *   yz_probe_cz case.toml out.bin parts    takes the pieces of one step on the
 *                                          start state instead, each written
 *                                          as the reference forms it: the
 *                                          film's assembly (SetMatrixA), its
 *                                          conservative update with h_new =
 *                                          h_old (the face fluxes), the
 *                                          velocity (CalVelocity) and the
 *                                          concentration's assembly
 *                                          (SetMatrixA) with those fluxes.
 *
 * out.bin is a list of named records: magic "YZCZREC1", then per record an
 * int32 name length, the name, an int32 kind (0 int32, 1 float64), an int64
 * count and the values (little endian).  tests/golden/stateio.py reads it.
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
#include "ConcZ_Model_2D.h"
#undef private
#undef protected

using namespace yuzen;

namespace {

struct Rec
{
	std::string name;
	int kind;
	std::vector<int> i;
	std::vector<double> d;
};
std::vector<Rec> g_recs;

void PutI(const std::string &n, const std::vector<int> &v) { g_recs.push_back(Rec{n, 0, v, {}}); }
void PutD(const std::string &n, const std::vector<double> &v) { g_recs.push_back(Rec{n, 1, {}, v}); }
void PutI(const std::string &n, int v) { PutI(n, std::vector<int>{v}); }
void PutD(const std::string &n, double v) { PutD(n, std::vector<double>{v}); }

bool Write(const char *path)
{
	FILE *f = std::fopen(path, "wb");
	if(!f) return false;
	std::fwrite("YZCZREC1", 1, 8, f);
	for(const Rec &r : g_recs)
	{
		const int len = (int)r.name.size();
		std::fwrite(&len, sizeof(int), 1, f);
		std::fwrite(r.name.data(), 1, r.name.size(), f);
		std::fwrite(&r.kind, sizeof(int), 1, f);
		const long long cnt = r.kind == 0 ? (long long)r.i.size() : (long long)r.d.size();
		std::fwrite(&cnt, sizeof(long long), 1, f);
		if(r.kind == 0) std::fwrite(r.i.data(), sizeof(int), r.i.size(), f);
		else std::fwrite(r.d.data(), sizeof(double), r.d.size(), f);
	}
	std::fclose(f);
	return true;
}

struct Probe
{
	ConcZ_Model_2D *m;
	C_Grid2D *G2;
	C_Grid3D *G3;
	int nx, ny, nz;

	std::vector<double> H() const
	{
		std::vector<double> v((size_t)nx * ny);
		for(int j = 0; j < ny; ++j)
			for(int i = 0; i < nx; ++i) v[(size_t)j * nx + i] = m->_field.HH(G2->At<Zface>(i, j));
		return v;
	}
	std::vector<double> S() const
	{
		std::vector<double> v((size_t)nx * ny);
		for(int j = 0; j < ny; ++j)
			for(int i = 0; i < nx; ++i) v[(size_t)j * nx + i] = m->_field.SS(G2->At<Zface>(i, j));
		return v;
	}
	std::vector<double> C() const
	{
		std::vector<double> v((size_t)nx * ny * nz);
		for(int k = 0; k < nz; ++k)
			for(int j = 0; j < ny; ++j)
				for(int i = 0; i < nx; ++i)
					v[((size_t)k * ny + j) * nx + i] = m->_field.CC(G3->At<Cell>(i, j, k));
		return v;
	}
	//  the in-plane velocity on the faces: face ix of a row (between ix-1 and
	//  ix), face jy of a column, at every level, in the layout of c
	std::vector<double> Ux() const
	{
		std::vector<double> v((size_t)nx * ny * nz);
		for(int k = 0; k < nz; ++k)
			for(int j = 0; j < ny; ++j)
				for(int i = 0; i < nx; ++i)
					v[((size_t)k * ny + j) * nx + i] = m->_field.Ux(G3->At<Xface>(i, j, k));
		return v;
	}
	std::vector<double> Uy() const
	{
		std::vector<double> v((size_t)nx * ny * nz);
		for(int k = 0; k < nz; ++k)
			for(int j = 0; j < ny; ++j)
				for(int i = 0; i < nx; ++i)
					v[((size_t)k * ny + j) * nx + i] = m->_field.Uy(G3->At<Yface>(i, j, k));
		return v;
	}
};

void PutPattern(const std::string &pre, const CRS_Matrix &A)
{
	const int n = A.RowSize(), nnz = A.NonZero();
	PutI(pre + "_rowptr", std::vector<int>(A.RowPtrData(), A.RowPtrData() + n + 1));
	PutI(pre + "_col", std::vector<int>(A.ColIndData(), A.ColIndData() + nnz));
	std::vector<int> flag((size_t)n);
	for(int i = 0; i < n; ++i) flag[(size_t)i] = A.IsBC(i) ? 1 : 0;
	PutI(pre + "_bc", flag);
}

std::vector<double> Values(const CRS_Matrix &A)
{
	std::vector<double> v;
	for(int r = 0; r < A.RowSize(); ++r)
		for(int j = 0; j < A.NonZero(r); ++j) v.push_back(A.Element(r, j));
	return v;
}

std::vector<double> Vec(const Vector<double> &x)
{
	std::vector<double> v((size_t)x.size());
	for(int i = 0; i < x.size(); ++i) v[(size_t)i] = x[i];
	return v;
}

} // namespace

int main(int argc, char **argv)
{
	if(argc < 3) { std::fprintf(stderr, "usage: yz_probe_cz case.toml out.bin [parts] [init=h.bin]\n"); return 2; }
	bool parts = false;
	const char *init = nullptr;
	for(int a = 3; a < argc; ++a)
	{
		if(std::strcmp(argv[a], "parts") == 0) parts = true;
		else if(std::strncmp(argv[a], "init=", 5) == 0) init = argv[a] + 5;
	}
	C_Yuzen solver;
	if(!solver.ReadInputFile(argv[1])) return 1;
	if(!solver.Initialize()) return 1;
	ConcZ_Model_2D *m = dynamic_cast<ConcZ_Model_2D*>(solver._model);
	if(!m) { std::fprintf(stderr, "yz_probe_cz: the case does not build the ConcZ model\n"); return 3; }
	Input &inp = *m->_inputParam;
	NonDimensionalNumbers &nd = m->_NonDim;
	//  the prologue of ConcZ_Model_2D::Run (ConcZ_Model_2D.cpp:714-735), which
	//  Run repeats: the step capped by the output intervals
	{
		double max_dt = m->_timeStep.MaxDT(), val;
		const double T0 = nd.TimeScale();
		if(!inp.Output.FieldData.Listed()) { val = inp.Output.FieldData.TimeInterval / T0; if(val < max_dt) max_dt = val; }
		val = inp.Output.ProbeList.TimeInterval / T0;		if(val < max_dt) max_dt = val;
		val = inp.Output.GeneralHistory.TimeInterval / T0;	if(val < max_dt) max_dt = val;
		val = inp.Output.CalcInfo.TimeInterval / T0;		if(val < max_dt) max_dt = val;
		m->_timeStep.SetMaxDT(max_dt);
		if(m->_timeStep.MaxDT() < m->_timeStep.DT().initial) m->_timeStep.ChangeDT(m->_timeStep.MaxDT());
	}
	Probe P;
	P.m = m;
	P.G2 = m->_field.GetGridPtr2();
	P.G3 = m->_field.GetGridPtr3();
	P.nx = P.G3->nx(); P.ny = P.G3->ny(); P.nz = P.G3->nz();
	auto &he = m->_heightEq;
	auto &ce = m->_concEq;
	const BoundaryCondition2D &bc = m->_boundary;
	if(init)
	{
		std::vector<double> h((size_t)P.nx * P.ny);
		FILE *f = std::fopen(init, "rb");
		if(!f || std::fread(h.data(), sizeof(double), h.size(), f) != h.size())
		{
			std::fprintf(stderr, "yz_probe_cz: cannot read %zu doubles from %s\n", h.size(), init);
			return 5;
		}
		std::fclose(f);
		for(int j = 0; j < P.ny; ++j)
			for(int i = 0; i < P.nx; ++i)
			{
				const double v = h[(size_t)j * P.nx + i];
				m->_field.HH(P.G2->At<Zface>(i, j)) = v;
				he._phi_old2[j * P.nx + i] = v;
				he._phi_old[j * P.nx + i] = v;
				he._phi_new[j * P.nx + i] = v;
			}
		he.TakeFieldAsStart();
	}

	PutI("nx", P.nx); PutI("ny", P.ny); PutI("nz", P.nz);
	PutI("bc", std::vector<int>{(int)bc._tXmin, (int)bc._tXmax, (int)bc._tYmin, (int)bc._tYmax});
	PutI("on_lap", he._sw_LaplacePressure ? 1 : 0);
	PutI("on_sc", he._sw_SolutoCapillarity ? 1 : 0);
	PutI("on_vg", he._sw_VerticalGravity ? 1 : 0);
	PutI("on_hg", he._sw_HorizontalGravity ? 1 : 0);
	PutI("on_cf", he._sw_Centrifugal ? 1 : 0);
	PutI("on_evap", nd._evap.Enabled() ? 1 : 0);
	PutI("on_mms", he._mms.Enabled() ? 1 : 0);
	PutI("ev_conc", (int)nd._evap._t_ConcFunc);
	PutI("ev_spatial", (int)nd._evap._t_SpatialFunc);
	PutI("ev_hast", nd._evap._sw_Hast_modify ? 1 : 0);
	PutI("dt_control", he._adjustTimeStep ? 1 : 0);
	PutI("dt_keep_steps", he._adjustTimeKeepSteps);
	PutI("max_steps", (int)inp.Numerics.MaxSteps);
	PutI("h_lin", std::vector<int>{(int)he._bcg._set.precondition, he._bcg._set.scaling ? 1 : 0,
	                               he._bcg._set.maxIteration, he._bcg._set.conc ? 1 : 0});
	PutI("c_lin", std::vector<int>{(int)ce._bcg._set.precondition, ce._bcg._set.scaling ? 1 : 0,
	                               ce._bcg._set.maxIteration, ce._bcg._set.conc ? 1 : 0});
	PutI("c_scheme", (int)ce._scheme.Scheme());

	PutD("dx", P.G3->dx()); PutD("dy", P.ny > 1 ? P.G3->dy() : 1.0); PutD("dzeta", P.G3->dz());
	PutD("theta_h", he._theta); PutD("theta_c", ce._theta);
	PutD("dt", m->_timeStep.DT().now); PutD("dt_old", m->_timeStep.DT().old);
	PutD("dt_max", m->_timeStep.DT().range_max); PutD("dt_min", m->_timeStep.DT().range_min);
	PutD("time", m->_timeStep.NowTime());
	PutD("dt_change_factor", he._adjustTimeChangeFactor); PutD("dt_criterion", he._adjustTimeCriterion);
	PutD("dt_scale_floor", he._adjustTimeScaleFloor);
	PutD("As", nd.As()); PutD("Ma", nd.Ma()); PutD("Bo", nd.Bo()); PutD("Pgx", nd.Pgx()); PutD("Pgy", nd.Pgy());
	PutD("Sp", nd.Sp()); PutD("Df", nd.Df()); PutD("Ev", nd.Ev());
	PutD("rot_center", std::vector<double>{he._rotCenter[0], he._rotCenter[1]});
	PutD("visc", std::vector<double>{nd._viscosity._baseConc, nd._viscosity._baseValue, nd._viscosity._exponent});
	PutD("sigma", std::vector<double>{nd._surface_tension._baseConc, nd._surface_tension._baseValue,
	                                  nd._surface_tension._coef});
	PutD("diff", std::vector<double>{nd._diffusivity._baseConc, nd._diffusivity._baseValue, nd._diffusivity._exponent});
	PutD("evap", std::vector<double>{nd._evap._M_resin, nd._evap._M_solvent, nd._evap._E0, nd._evap._powerN,
	                                 nd._evap._NegPowExponent, nd._evap._NegPowRmax, nd._evap._ConcR, nd._evap._h_ast,
	                                 std::min(nd._evap._G.dx(), nd._evap._G.dy())});
	PutD("h_eps", he._bcg._set.epsilon); PutD("c_eps", ce._bcg._set.epsilon);
	PutD("coupling_floor", he._couplingFloor);
	{
		std::vector<double> xc((size_t)P.nx), xf((size_t)P.nx), yc((size_t)P.ny), yf((size_t)P.ny);
		for(int i = 0; i < P.nx; ++i)
		{
			xc[(size_t)i] = P.G2->X(P.G2->At<Zface>(i, 0));
			xf[(size_t)i] = P.G2->XOf<Yedge>(i, 0);
		}
		for(int j = 0; j < P.ny; ++j)
		{
			yc[(size_t)j] = P.G2->Y(P.G2->At<Zface>(0, j));
			yf[(size_t)j] = P.ny > 1 ? P.G2->YOf<Xedge>(0, j) : 0.0;
		}
		PutD("xc", xc); PutD("xf", xf); PutD("yc", yc); PutD("yf", yf);
	}
	PutD("h0", P.H()); PutD("s", P.S()); PutD("c0", P.C());
	PutPattern("h", he._crsA);
	PutPattern("c", ce._crsA);

	if(parts)
	{
		//  the film's assembly of the start state at the step's dt
		he.EveryTimeStepTrial();
		he.SetMatrixA();
		PutD("h_A", Values(he._crsA)); PutD("h_B", Vec(he._VecB));
		PutD("h_colsrc", he._colSrc);
		PutD("h_qcapx", he._qCapX); PutD("h_qexpx", he._qExpX);
		PutD("h_qcapy", he._qCapY); PutD("h_qexpy", he._qExpY);
		he.MakeMatrix_IA();
		PutD("h_IA", Values(he._crsIA));
		//  the conservative update of an unchanged film: the face fluxes of
		//  h_old and the end of the step through them
		he._phi_old = he._phi_new;
		he.ConservativeUpdate();
		PutD("h_qx", he._qX); PutD("h_qy", he._qY); PutD("h_end", Vec(he._phi_new));
		he.CalDtDh();
		PutD("h_dtdh", Vec(he._dtdh));
		ce.SetDtDh(he.GetDtDh());
		he.CalVelocity();
		PutD("ux", P.Ux()); PutD("uy", P.Uy());
		ce.SetMatrixA();
		PutD("c_A", Values(ce._crsA)); PutD("c_B", Vec(ce._VecB)); PutD("c_rhs", Vec(ce._Rhs));
		PutD("c_react", ce._react);
		PutD("c_qx", ce._Qx); PutD("c_qy", ce._Qy); PutD("c_w", ce._W);
	}
	else
	{
		auto t0 = std::chrono::steady_clock::now();
		m->Run();
		auto t1 = std::chrono::steady_clock::now();
		solver.Finalize();
		PutD("wall", std::chrono::duration<double>(t1 - t0).count());
		PutD("t_end", m->_timeStep.NowTime());
		PutD("dt_end", m->_timeStep.DT().now);
		PutI("steps_done", (int)m->_nSteps);
		PutI("linear_iterations", (int)m->_sumBCGIter);
		PutI("coupling_passes", (int)m->_sumCoupling);
		PutI("diverged", m->Diverged() ? 1 : 0);
		PutD("h1", P.H()); PutD("c1", P.C());
	}
	return Write(argv[2]) ? 0 : 4;
}
