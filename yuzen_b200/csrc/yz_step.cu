// yz_step.cu -- the implicit step of the well-mixed film-height equation on
// the device: assembly of A, J, I + theta dt J and the right-hand side for
// every enabled term, the Newton-Kantorovich loop (NewtonKantorovich.cpp:
// 157-486) and the time-step control (ImplicitSolver.cpp:144-190, 271-307),
// around the device linear solve of yz_solver.cu.
#include "yz_physics.cuh"
#include "yz_upwind.cuh"
#include "yz_conc.cuh"
#include "yz_step_impl.h"
#include "yz_prof.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>

namespace yz {

using namespace phys;

namespace {

__device__ __forceinline__ int Offset(int s, int nx)
{
	switch(s)
	{
	case oM: return -2 * nx;
	case mm: return -nx - 1;
	case om: return -nx;
	case pm: return -nx + 1;
	case Mo: return -2;
	case mo: return -1;
	case oo: return 0;
	case po: return 1;
	case Po: return 2;
	case mp: return nx - 1;
	case op: return nx;
	case pp: return nx + 1;
	default: return 2 * nx;
	}
}

//  |v| into a running maximum: non-negative doubles order as their bit
//  patterns, so the warp's maximum goes in with one integer atomicMax
__device__ __forceinline__ void WarpMaxAbs(unsigned long long *slot, double v)
{
	unsigned long long u = (unsigned long long)__double_as_longlong(fabs(v));
	for(int off = 16; off >= 1; off >>= 1)
	{
		const unsigned long long w = __shfl_down_sync(0xffffffffu, u, off);
		u = w > u ? w : u;
	}
	if((threadIdx.x & 31) == 0 && u) atomicMax(slot, u);
}

//--------------------------------------------------------------------------
//  Face properties (FaceBuf): one thread per face; with J, also the
//  derivatives the Jacobian takes.  Faces of axis x: low cells ix 1..nx-3,
//  iy 2..ny-3; of axis y: ix 2..nx-3, iy 1..ny-3.
//--------------------------------------------------------------------------
template<bool J>
__global__ void KFaceProps(Coef k, const double *__restrict__ H, const double *__restrict__ C, FaceBuf fb)
{
	const int nx = k.nx, ny = k.ny;
	const int nxF = (nx - 3) * (ny - 4), nyF = (nx - 4) * (ny - 3);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nxF + nyF; t += gridDim.x * blockDim.x)
	{
		int lo, hi;
		FaceSet f;
		bool pinned;
		if(t < nxF)
		{
			const int ix = 1 + t % (nx - 3), iy = 2 + t / (nx - 3);
			lo = iy * nx + ix; hi = lo + 1; f = fb.x;
			pinned = (ix == 1 && k.pinned[0]) || (ix == nx - 3 && k.pinned[1]);
		}
		else
		{
			const int u = t - nxF;
			const int ix = 2 + u % (nx - 4), iy = 1 + u / (nx - 4);
			lo = iy * nx + ix; hi = lo + nx; f = fb.y;
			pinned = (iy == 1 && k.pinned[2]) || (iy == ny - 3 && k.pinned[3]);
		}
		const double hl = H[lo], hh = H[hi];
		const double cfc = 0.5 * (C[lo] + C[hi]);
		const double vis = Viscosity(k, cfc), sig = SurfaceTension(k, cfc);
		const double FM = Face(k, hl, hh);
		const double val = k.slip ? FM : 2.0 * (hl * hl) * (hh * hh) / (hl + hh);
		f.vis[lo] = vis; f.sig[lo] = sig; f.FM[lo] = FM;
		//  LaplacePressure_WM2D::PinnedFace (LaplacePressure_2D.cpp:21-30): the
		//  capillary term's mobility and its derivatives zero on a pinned face
		f.DL[lo] = pinned ? 0.0 : val * sig / vis;
		if(!J) continue;
		const double dLH = (k.onV || k.onD || k.slip) ? Face_d1(k, hl, hh) : 0.0;
		const double dHL = (k.onV || k.onD || k.slip) ? Face_d1(k, hh, hl) : 0.0;
		f.fdLH[lo] = dLH; f.fdHL[lo] = dHL;
		if(k.onL)
		{
			//  NonlinearJacobiProps (LaplacePressureKernel.h:160-175)
			const double den = (hl + hh) * (hl + hh);
			const double vLH = k.slip ? dLH : 2.0 * (hl * hh * hh) * (hl + hh + hh) / den;
			const double den2 = (hh + hl) * (hh + hl);
			const double vHL = k.slip ? dHL : 2.0 * (hh * hl * hl) * (hh + hl + hl) / den2;
			f.gLH[lo] = pinned ? 0.0 : vLH * sig / vis;
			f.gHL[lo] = pinned ? 0.0 : vHL * sig / vis;
		}
	}
}

//  Pi, Pi / h and dPi of every cell (DisjoiningPressureKernel.h:191-218),
//  from one pair of pow calls
__global__ void KCellPi(Coef k, int n, const double *__restrict__ H, FaceBuf fb)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double hj = H[i];
		if(hj <= 0) { fb.piN[i] = 0; fb.phN[i] = 0; fb.dpN[i] = 0; continue; }
		const double r = k.hstar / hj;
		const double rn = pow(r, k.pn), rm = pow(r, k.pm);
		const double p = rn - rm;
		fb.piN[i] = p;
		fb.phN[i] = p / hj;
		fb.dpN[i] = -(k.pn * rn - k.pm * rm) / hj;
	}
}

//  face d of the interior row i: its index in the face arrays and whether
//  the row is the face's low cell
__device__ __forceinline__ void FaceOf(int d, int i, int nx, const FaceBuf &fb, FaceSet &f, int &idx, bool &low)
{
	switch(d)
	{
	case 0:  f = fb.x; idx = i - 1; low = false; break;
	case 1:  f = fb.x; idx = i; low = true; break;
	case 2:  f = fb.y; idx = i - nx; low = false; break;
	default: f = fb.y; idx = i; low = true; break;
	}
}

//--------------------------------------------------------------------------
//  The limited upwind terms' faces (UpwindFaces in yz_upwind.cuh): one
//  thread a cell and (grid y) an axis and a term, the cell's high face on
//  that axis where a row needs it
//--------------------------------------------------------------------------
template<bool J>
__global__ void KUpwindFaces(Coef k, const double *__restrict__ H, const double *__restrict__ C, FaceBuf fb,
                             UpBuf up)
{
	const int a = blockIdx.y / 3, term = blockIdx.y % 3;
	if(!(term == 0 ? k.onPG : term == 1 ? k.onCF : k.onSC)) return;
	const int nx = k.nx, ny = k.ny;
	const long long n = (long long)nx * ny;
	const long long s = (a == 0) ? 1 : nx;
	for(long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
	{
		const int ix = (int)(j % nx), iy = (int)(j / nx);
		const bool in = (a == 0) ? (ix >= 1 && ix <= nx - 3 && iy >= 2 && iy <= ny - 3)
		                         : (iy >= 1 && iy <= ny - 3 && ix >= 2 && ix <= nx - 3);
		if(!in) continue;
		const double f[4] = {H[j - s], H[j], H[j + s], H[j + 2 * s]};
		const double vis = (a == 0) ? fb.x.vis[j] : fb.y.vis[j];
		const bool wall = WallFaceLow(k, a, ix, iy);
		if(term == 0) BodyForceFace<kPG, J>(k, f, vis, a, ix, iy, wall, up, j);
		else if(term == 1) BodyForceFace<kCF, J>(k, f, vis, a, ix, iy, wall, up, j);
		else MarangoniFace<J>(k, f, C[j], C[j + s], vis, a, wall, up, j);
	}
}

//--------------------------------------------------------------------------
//  One interior row: the A entries of every term, then what the caller
//  asks for: mode 0 -> A(h) h only (the explicit half and evapOld);
//  mode 1 -> I + theta dt J, A(h) h, B and the right-hand side.
//--------------------------------------------------------------------------
struct RowOut
{
	double *ia;        // values of I + theta dt J (storage order)
	double *ax;        // A(h) h
	double *evapOld;   // mode 0: written; mode 1: read
	double *evapB;     // mode 1: the evaporation B took
	double *rhs;       // mode 1
	const double *hOld, *axOld;
	unsigned long long *rhsMax;
	const double *src;   // mode 1: the nozzle's supply of the step, or null
};

//  three blocks of 128 a SM (168 registers a thread, a few spills) ran the
//  512^2 all-physics assembly 13 % faster than two (255 registers); four or
//  five blocks spill more than the occupancy gains
#ifndef YZ_ASSEMBLE_MIN_BLOCKS
#define YZ_ASSEMBLE_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(128, YZ_ASSEMBLE_MIN_BLOCKS)
KAssemble(Coef k, int mode, double dt, const int *__restrict__ rowptr,
                          const double *__restrict__ H, const double *__restrict__ C,
                          const double *__restrict__ S, RowOut o, FaceBuf fb, UpBuf up)
{
	const int nx = k.nx, ny = k.ny;
	const int nIn = (nx - 4) * (ny - 4);
	double rmax = 0.0;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nIn; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		double h[13], c[13], s[13];
#pragma unroll
		for(int q = 0; q < 13; ++q)
		{
			const int j = i + Offset(q, nx);
			h[q] = H[j]; c[q] = C[j]; s[q] = S[j];
		}
		const double hoo = h[oo], coo = c[oo];
		//  face properties
		(void)coo;
		double vis[4], DL[4], FM[4], Haj[4];
		int fIdx[4];
		bool fLow[4];
		FaceSet fs[4];
#pragma unroll
		for(int d = 0; d < 4; ++d)
		{
			Haj[d] = h[AdjIdx(d)];
			FaceOf(d, i, nx, fb, fs[d], fIdx[d], fLow[d]);
			vis[d] = fs[d].vis[fIdx[d]];
			FM[d] = fs[d].FM[fIdx[d]];
			DL[d] = fs[d].DL[fIdx[d]];
		}
		double aA[13], aR[13];
#pragma unroll
		for(int q = 0; q < 13; ++q) { aA[q] = 0.0; aR[q] = 0.0; }
		//  --- LaplacePressureKernel::SetMatrixA (LaplacePressureKernel.h:354-433)
		if(k.onL)
		{
			double Tf[4];
#pragma unroll
			for(int d = 0; d < 4; ++d) Tf[d] = DL[d] / hoo;
			double topo = 0;
#pragma unroll
			for(int q = 0; q < 13; ++q)
			{
				double cc = 0;
#pragma unroll
				for(int d = 0; d < 4; ++d) cc += k.cL[d][q] * Tf[d];
				topo += cc * s[q];
			}
#pragma unroll
			for(int q = 0; q < 13; ++q)
			{
				double val = 0;
#pragma unroll
				for(int d = 0; d < 4; ++d) val += k.cL[d][q] * DL[d];
				if(q == oo) val += topo;
				aA[q] += k.coefL * val;
			}
		}
		//  --- VerticalGravityKernel::SetMatrixA (VerticalGravityKernel.h)
		double G[4], Tface[4];
#pragma unroll
		for(int d = 0; d < 4; ++d)
		{
			G[d] = FM[d] / vis[d];
			Tface[d] = (FM[d] == 0) ? 0.0 : FM[d] / (hoo + Haj[d]) / vis[d];
		}
		if(k.onV)
		{
			double Tsum[4], Too = 0;
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				Tsum[d] = 0;
#pragma unroll
				for(int q = 0; q < 13; ++q) Tsum[d] += k.cG[d][q] * s[q];
			}
#pragma unroll
			for(int kk = 0; kk < 4; ++kk) { const int dd = StencilDir(kk); Too += Tsum[dd] * Tface[dd]; }
#pragma unroll
			for(int d = 0; d < 4; ++d) Tsum[d] *= Tface[d];
#pragma unroll
			for(int kk = 0; kk < 5; ++kk)
			{
				const int idx = NarrowIdx(kk);
				double val = 0;
#pragma unroll
				for(int d = 0; d < 4; ++d) val += k.cG[d][idx] * G[d];
				if(idx == oo) val += Too;
				else val += Tsum[DirOfAdj(idx)];
				aA[idx] += k.coefV * val;
			}
		}
		//  --- the upwinded terms into A_rest, in the order of the physics list
		//  (HeightEquationBase.h:565-577): in-plane gravity, Marangoni, rotation
		if(k.onPG) BodyForceAF<kPG>(k, up, i, aR);
		if(k.onSC) MarangoniAF(k, up, i, aR);
		if(k.onCF) BodyForceAF<kCF>(k, up, i, aR);
		//  --- DisjoiningPressureKernel::SetMatrixA (DisjoiningPressureKernel.h:306-349).
		//  Pi, Pi/h and dPi of the five narrow points from one pair of pow
		//  calls each: the same values the reference's three functions give
		double piN[13], phN[13], dpN[13];
		if(k.onD)
		{
#pragma unroll
			for(int kk = 0; kk < 5; ++kk)
			{
				const int idx = NarrowIdx(kk);
				const int j = i + Offset(idx, nx);
				piN[idx] = fb.piN[j]; phN[idx] = fb.phN[j]; dpN[idx] = fb.dpN[j];
			}
#pragma unroll
			for(int kk = 0; kk < 5; ++kk)
			{
				const int idx = NarrowIdx(kk);
				const double php = phN[idx];
				double val = 0;
#pragma unroll
				for(int d = 0; d < 4; ++d) val += k.cG[d][idx] * G[d];
				val *= php;
				aR[idx] += k.coefD * val;
			}
		}
		//  A = A + A_rest (HeightEquationBase.h:749-759)
		double A[13];
#pragma unroll
		for(int q = 0; q < 13; ++q) A[q] = aA[q] + aR[q];

		//  --- ApplyA (HeightEquationBase.h:804-827): A_rest h in storage
		//  order, then the conservative fluxes of the capillary and the
		//  vertical gravity terms
		double y = 0.0;
		y = y + aR[oo] * h[oo];
		for(int q = 0; q < 13; ++q) if(q != oo) y = y + aR[q] * h[q];
		if(k.onL)
		{
			double r = 0;
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				const double f = k.coefL * (DL[d] * (FaceGradient(k, h, d) + FaceGradient(k, s, d)));
				r += (d % 2 == 0) ? -f : f;
			}
			y += r;
		}
		if(k.onV)
		{
			double r = 0;
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				const int a = AdjIdx(d);
				const double hl = (d % 2 == 0) ? h[a] : hoo, hh = (d % 2 == 0) ? hoo : h[a];
				const double sl = (d % 2 == 0) ? s[a] : s[oo], sh = (d % 2 == 0) ? s[oo] : s[a];
				const double dn = (d < 2) ? k.dxx : k.dyy;
				const double mu = vis[d];
				double gf = Face(k, hl, hh);
				const double tk = (gf == 0) ? 0.0 : gf / (hl + hh) / mu;
				gf /= mu;
				const double f = k.coefV * ((gf * (hh - hl) + (sh - sl) * (tk * (hl + hh))) / (dn * dn));
				r += (d % 2 == 0) ? -f : f;
			}
			y += r;
		}
		o.ax[i] = y;

		//  the cell centre (RectGrid::X of a cell site, RectGrid.h:375-383)
		const double xx = k.xmin + ix * k.dx + k.dx2h, yy = k.ymin + iy * k.dy + k.dy2h;
		if(mode == 0)
		{
			if(k.onEvap) o.evapOld[i] = EvapAt(k, hoo, coo, xx, yy, dt);
			continue;
		}

		//  --- SetMatrixJacobi (HeightEquationBase.h:1062-1091): J = A, then
		//  every term's Jacobian
		double J[13];
#pragma unroll
		for(int q = 0; q < 13; ++q) J[q] = A[q];
		//  the face mobility's derivatives by the neighbour (A) and by this
		//  cell (C): Mobility::Face_d1, which with slip is also the capillary
		//  term's FaceDK_d1; evaluated once for every term
		double fdA[4], fdC[4];
#pragma unroll
		for(int d = 0; d < 4; ++d)
		{
			const double LH = fs[d].fdLH[fIdx[d]], HL = fs[d].fdHL[fIdx[d]];
			fdA[d] = fLow[d] ? HL : LH;
			fdC[d] = fLow[d] ? LH : HL;
		}
		if(k.onL)
		{
			double a[4], b[4], gAdj[4], gCen[4], sAdj[4], sCen[4];
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				a[d] = 0; b[d] = 0;
#pragma unroll
				for(int q = 0; q < 13; ++q) { a[d] += k.cL[d][q] * h[q]; b[d] += k.cL[d][q] * s[q]; }
				//  NonlinearJacobiProps (LaplacePressureKernel.h:160-175), by
				//  the neighbour and by this cell
				{
					const double LH = fs[d].gLH[fIdx[d]], HL = fs[d].gHL[fIdx[d]];
					gAdj[d] = fLow[d] ? HL : LH;
					gCen[d] = fLow[d] ? LH : HL;
				}
				sAdj[d] = gAdj[d] / hoo;
				sCen[d] = gCen[d] / hoo - DL[d] / (hoo * hoo);
			}
			double gaSum = 0, sbSum = 0;
#pragma unroll
			for(int kk = 0; kk < 4; ++kk) { const int dd = StencilDir(kk); gaSum += gCen[dd] * a[dd]; }
#pragma unroll
			for(int d = 0; d < 4; ++d) sbSum += sCen[d] * b[d];
#pragma unroll
			for(int kk = 0; kk < 5; ++kk)
			{
				const int idx = NarrowIdx(kk);
				if(idx == oo) J[oo] += k.coefL * (gaSum + sbSum * hoo);
				else
				{
					const int dd = DirOfAdj(idx);
					J[idx] += k.coefL * (gAdj[dd] * a[dd] + sAdj[dd] * b[dd] * hoo);
				}
			}
		}
		if(k.onV)
		{
			double a[4], b[4], gAdj[4], gCen[4];
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				a[d] = 0; b[d] = 0;
#pragma unroll
				for(int q = 0; q < 13; ++q) { a[d] += k.cG[d][q] * h[q]; b[d] += k.cG[d][q] * s[q]; }
				gAdj[d] = fdA[d] / vis[d];
				gCen[d] = fdC[d] / vis[d];
			}
			double gaSum = 0;
#pragma unroll
			for(int kk = 0; kk < 4; ++kk)
			{
				const int dd = StencilDir(kk);
				gaSum += gCen[dd] * (a[dd] + b[dd]) - Tface[dd] * b[dd];
			}
#pragma unroll
			for(int kk = 0; kk < 5; ++kk)
			{
				const int idx = NarrowIdx(kk);
				if(idx == oo) J[oo] += k.coefV * gaSum;
				else
				{
					const int dd = DirOfAdj(idx);
					J[idx] += k.coefV * (gAdj[dd] * (a[dd] + b[dd]) - Tface[dd] * b[dd]);
				}
			}
		}
		if(k.onPG) BodyForceJF<kPG>(k, up, i, J);
		if(k.onSC) MarangoniJF(k, up, i, J);
		if(k.onCF) BodyForceJF<kCF>(k, up, i, J);
		if(k.onD)
		{
			double Ad[4], gAdj[4], gCen[4];
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				//  only the two non-zero coefficients, in stencil-point order
				const int a = AdjIdx(d);
				const int lo = a < oo ? a : oo, hi = a < oo ? oo : a;
				double acc = 0;
				acc += k.cG[d][lo] * piN[lo];
				acc += k.cG[d][hi] * piN[hi];
				Ad[d] = acc;
				gAdj[d] = fdA[d] / vis[d];
				gCen[d] = fdC[d] / vis[d];
			}
			double gaSum = 0, gcSum = 0;
#pragma unroll
			for(int kk = 0; kk < 4; ++kk)
			{
				const int dd = StencilDir(kk);
				gaSum += gCen[dd] * Ad[dd];
				gcSum += G[dd] * k.cG[dd][oo];
			}
#pragma unroll
			for(int kk = 0; kk < 5; ++kk)
			{
				const int idx = NarrowIdx(kk);
				const double dpi = dpN[idx] - phN[idx];
				if(idx == oo) J[oo] += k.coefD * (gaSum + gcSum * dpi);
				else
				{
					const int dd = DirOfAdj(idx);
					J[idx] += k.coefD * (gAdj[dd] * Ad[dd] + G[dd] * k.cG[dd][idx] * dpi);
				}
			}
		}
		//  --- MakeMatrix_IA (NewtonKantorovich.cpp:488-510)
		const int base = rowptr[i];
		const double td = k.theta * dt;
		o.ia[base] = 1.0 + td * J[oo];
#pragma unroll
		for(int q = 0; q < 13; ++q) if(q != oo) o.ia[base + Pos(q)] = td * J[q];
		//  --- B (HeightEquationBase.h:771-787) and MakeRHS (:512-523)
		double evp = 0.0;
		if(k.onEvap) evp = (1.0 - k.theta) * o.evapOld[i] + k.theta * EvapAt(k, hoo, coo, xx, yy, dt);
		o.evapB[i] = evp;
		const double B = evp - (o.src ? o.src[i] : 0.0);
		const double r = o.hOld[i] - hoo - (dt * k.theta * y) - (dt * (1.0 - k.theta) * o.axOld[i]) - dt * B;
		o.rhs[i] = r;
		rmax = fmax(rmax, fabs(r));
	}
	if(mode == 1) WarpMaxAbs(o.rhsMax, rmax);
}

//--------------------------------------------------------------------------
//  The energy budget (EnergyBudget.h; WellMixedModelBase.h:883-893): the
//  free energy F = sum over the real cells of Bo/2 f^2 + Dp w(h) plus the
//  capillary energy of the cell's high faces (and of its low faces on an
//  edge that is not periodic), f = h + s, times dx dy; and the flux power
//  D = sum over the real cells of phi (-div F) times dx dy
//  (HeightEquationBase::FluxPower with no side rate in 2-D), phi the
//  driving potential (LubFields.cpp:278-289) and F the face volume fluxes of
//  the film (FaceVolumeFluxes, KFaceFlux).  One element a thread over the
//  real cells, both sums by the fixed reduction tree.
//--------------------------------------------------------------------------
struct EnergyPar
{
	double bo, dp, hstar, pn, pm;
	int capillary, perX, perY;
};

//  w(h) = -int_{h*}^{h} Pi(s) ds (EnergyBudget.h:59-67)
__device__ __forceinline__ double EnergyW(const EnergyPar &e, double h)
{
	if(e.dp == 0 || !(h > 0)) return 0;
	const double hs = e.hstar, n = e.pn, m = e.pm;
	const double in = pow(hs, n) * (pow(h, 1.0 - n) - pow(hs, 1.0 - n)) / (1.0 - n);
	const double im = pow(hs, m) * (pow(h, 1.0 - m) - pow(hs, 1.0 - m)) / (1.0 - m);
	return -e.dp * (in - im);
}

__device__ __forceinline__ double EnergyFace(const Coef &k, const EnergyPar &e, double fi, double fj, double ci,
                                             double cj, double dn)
{
	if(!e.capillary) return 0;
	const double g = (fj - fi) / dn;
	return 0.25 * (SurfaceTension(k, ci) + SurfaceTension(k, cj)) * g * g;
}

__global__ void KEnergy(Coef k, EnergyPar e, const double *__restrict__ H, const double *__restrict__ C,
                        const double *__restrict__ S, const double *__restrict__ Fx, const double *__restrict__ Fy,
                        RedScratch rs, double *__restrict__ out)
{
	__shared__ double sh[2 * kRT];
	const int nx = k.nx, ny = k.ny;
	const int nIn = (nx - 4) * (ny - 4);
	const double dx2 = k.dx * k.dx, dy2 = k.dy * k.dy;
	double a[2] = {0.0, 0.0};
	for(int kk = 0, t = blockIdx.x * kRChunk + threadIdx.x; kk < kRK; ++kk, t += kRT)
	{
		if(t >= nIn) break;
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		const double h = H[i], c = C[i], v = H[i] + S[i];
		const double vxp = H[i + 1] + S[i + 1], vxm = H[i - 1] + S[i - 1];
		const double vyp = H[i + nx] + S[i + nx], vym = H[i - nx] + S[i - nx];
		//  FreeEnergy: the cell, its high faces, its low faces at a wall
		double f = 0.5 * e.bo * v * v + EnergyW(e, h);
		f = f + EnergyFace(k, e, v, vxp, c, C[i + 1], k.dx);
		f = f + EnergyFace(k, e, v, vyp, c, C[i + nx], k.dy);
		if(!e.perX && ix == 2) f = f + EnergyFace(k, e, vxm, v, C[i - 1], c, k.dx);
		if(!e.perY && iy == 2) f = f + EnergyFace(k, e, vym, v, C[i - nx], c, k.dy);
		//  Potential (PotentialAt) and FluxPower
		const double lap = (vxp - 2.0 * v + vxm) / dx2 + (vyp - 2.0 * v + vym) / dy2;
		double phi = 0;
		if(e.capillary) phi += SurfaceTension(k, c) * lap;
		if(e.dp != 0 && h > 0)
		{
			const double r = e.hstar / h;
			phi += e.dp * (pow(r, e.pn) - pow(r, e.pm));
		}
		if(e.bo != 0) phi -= e.bo * v;
		double div = 0;
		div += Fx[i] - Fx[i - 1];
		div += Fy[i] - Fy[i - nx];
		a[0] = a[0] + f;
		a[1] = a[1] + phi * (-div - 0.0);
	}
	double tot[2];
	if(GridFold<2>(a, sh, rs, tot) && threadIdx.x == 0)
	{
		out[0] = tot[0] * k.dx * k.dy;
		out[1] = tot[1] * (k.dx * k.dy);
	}
}

//  ghost rows of x satisfied exactly (CRS_Matrix::SatisfyBCRows for rows
//  [1, -1] with right-hand side 0: x_ghost = x_partner)
__global__ void KGhostCopy(int nGhost, const int *__restrict__ ghost, const int *__restrict__ partner,
                           double *__restrict__ x)
{
	for(int g = blockIdx.x * blockDim.x + threadIdx.x; g < nGhost; g += gridDim.x * blockDim.x)
		x[ghost[g]] = x[partner[g]];
}

__global__ void KAbsMax(int n, const double *__restrict__ x, unsigned long long *out)
{
	double m = 0.0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmax(m, fabs(x[i]));
	WarpMaxAbs(out, m);
}

//  phi += delta * alpha (Vector operator+= with Vector * scalar)
__global__ void KAxpyAlpha(int n, const double *__restrict__ d, double alpha, double *__restrict__ phi)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) phi[i] += d[i] * alpha;
}

//  opt extrap (NewtonKantorovich.cpp:179-198): g = phi + r (phi - phi2);
//  ok stays 1 unless a non-ghost cell with liquid would lose it; move = |g - phi|max
__global__ void KExtrapCheck(int n, const double *__restrict__ phi, const double *__restrict__ phi2,
                             const unsigned char *__restrict__ isbc, double r, int *notOk, unsigned long long *move)
{
	double m = 0.0;
	int bad = 0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double g = phi[i] + r * (phi[i] - phi2[i]);
		if(!isbc[i] && phi[i] > 0 && !(g > 0)) bad = 1;
		m = fmax(m, fabs(g - phi[i]));
	}
	if(bad) atomicExch(notOk, 1);
	WarpMaxAbs(move, m);
}

__global__ void KExtrapApply(int n, const double *__restrict__ phi, const double *__restrict__ phi2, double r,
                             double *__restrict__ guess)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		guess[i] = phi[i] + r * (phi[i] - phi2[i]);
}

//  LocalTruncationCriterion (ImplicitSolver.cpp:271-307): max |E_k|
__global__ void KLte(int n, const double *__restrict__ hp, const double *__restrict__ ho, const double *__restrict__ hm,
                     double dt0, double dt, double wfloor, unsigned long long *out)
{
	double m = 0.0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		double w = fabs(ho[i]);
		if(w < wfloor) w = wfloor;
		const double denom = (dt0 + dt) * w;
		const double e = (fabs(denom) <= 2.2250738585072014e-308)   // Math::IsZero
		    ? 0.0 : 2.0 * (dt / dt0) * (dt0 * hp[i] + dt * hm[i] - (dt0 + dt) * ho[i]) / denom;
		m = fmax(m, fabs(e));
	}
	WarpMaxAbs(out, m);
}

//  The nozzle's supply of every real cell (Source_WM2D::updateFraction and
//  operator(), WM2D/Source.cpp:40-110): the flow rate times the fraction of
//  the cell's sub^2 sample points within the nozzle's radius, for the cells
//  whose centre lies within the radius and a cell diagonal of the nozzle
__global__ void KSource(Coef k, double xn, double yn, double radius, int sub, double flow, double *__restrict__ src)
{
	const int nx = k.nx, n = nx * k.ny;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const int ix = i % nx, iy = i / nx;
		const double xc = k.xmin + ix * k.dx + k.dx2h, yc = k.ymin + iy * k.dy + k.dy2h;
		const double ex = xc - xn, ey = yc - yn;
		const double rr = sqrt(ex * ex + ey * ey);
		double alpha = 0.0;
		if(rr < radius + sqrt(k.dx * k.dx + k.dy * k.dy))
		{
			const double dxs = k.dx / (double)sub, dys = k.dy / (double)sub;
			const double xL = xc - 0.5 * k.dx, yB = yc - 0.5 * k.dy;
			for(int a = 0; a < sub; ++a)
			{
				const double xx = xL + ((double)a + 0.5) * dxs;
				for(int b = 0; b < sub; ++b)
				{
					const double yy = yB + ((double)b + 0.5) * dys;
					const double fx = xx - xn, fy = yy - yn;
					const double r2 = sqrt(fx * fx + fy * fy);
					alpha += (r2 <= radius ? 1.0 : 0.0);
				}
			}
			alpha /= (double)(sub * sub);
		}
		src[i] = flow * alpha;
	}
}

//  the right-hand side of the concentration's correction d on the ghost rows:
//  the row's b less its product with c0, summed in storage order
//  (ConcEquationBase.h:283-294)
__global__ void KBcRhs(int nGhost, const int *__restrict__ ghost, const int *__restrict__ rowptr,
                       const int *__restrict__ col, const double *__restrict__ val, const double *__restrict__ b,
                       const double *__restrict__ c0, double *__restrict__ rhs)
{
	for(int g = blockIdx.x * blockDim.x + threadIdx.x; g < nGhost; g += gridDim.x * blockDim.x)
	{
		const int i = ghost[g];
		double v = 0;
		for(int k = rowptr[i]; k < rowptr[i + 1]; ++k) v += val[k] * c0[col[k]];
		rhs[i] = b[g] - v;
	}
}

//  the ghosts of the concentration's d where every ghost copies one cell
//  (SatisfyBCRows of rows [1, -1] with the d system's right-hand side)
__global__ void KGhostD(int nGhost, const int *__restrict__ ghost, const int *__restrict__ partner,
                        const double *__restrict__ rhsD, double *__restrict__ d)
{
	for(int g = blockIdx.x * blockDim.x + threadIdx.x; g < nGhost; g += gridDim.x * blockDim.x)
	{
		const int i = ghost[g];
		d[i] = (rhsD[i] - (-1.0 * d[partner[g]])) / 1.0;
	}
}

//  y = a + d
__global__ void KAddTo(int n, const double *__restrict__ a, const double *__restrict__ d, double *__restrict__ y)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a[i] + d[i];
}

//  the Newton matrix's ghost rows and their right-hand side, once (yz_bc.h)
__global__ void KSetGhostRows(int nVal, const int *__restrict__ pos, const double *__restrict__ val, int nGhost,
                              const int *__restrict__ ghost, const double *__restrict__ grhs, double *__restrict__ ia,
                              double *__restrict__ rhs)
{
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nVal; t += gridDim.x * blockDim.x) ia[pos[t]] = val[t];
	for(int g = blockIdx.x * blockDim.x + threadIdx.x; g < nGhost; g += gridDim.x * blockDim.x) rhs[ghost[g]] = grhs[g];
}

//  CRS_Matrix::SatisfyBCRows (CRS_Matrix.cpp:198-302) on x with the plan of
//  yz_bc.h, one thread a set of coupled ghost rows: each row's right-hand
//  side less its other terms (in the plan's order), the elimination of the
//  right-hand side with the plan's pivots and multipliers, and the back
//  substitution on the eliminated matrix
__global__ void KSatisfyBC(BcSets S, double *__restrict__ x)
{
	for(int c = blockIdx.x * blockDim.x + threadIdx.x; c < S.n; c += gridDim.x * blockDim.x)
	{
		const int m = S.m[c];
		if(m <= 0 || m > kMaxBcSet) continue;
		const int r0 = S.rowOff[c], m0 = S.matOff[c];
		double b[kMaxBcSet];
		for(int p = 0; p < m; ++p)
		{
			double s = 0;
			for(int t = S.termOff[r0 + p]; t < S.termOff[r0 + p + 1]; ++t) s += S.termVal[t] * x[S.termCol[t]];
			b[p] = (S.rhsVec ? S.rhsVec[S.row[r0 + p]] : S.rhs[r0 + p]) - s;
		}
		for(int col = 0; col < m; ++col)
		{
			const int pv = S.piv[r0 + col];
			if(pv != col) { const double t = b[pv]; b[pv] = b[col]; b[col] = t; }
			for(int p = col + 1; p < m; ++p)
			{
				const double f = S.fac[m0 + p * m + col];
				if(f == 0.0) continue;
				b[p] -= f * b[col];
			}
		}
		for(int p = m - 1; p >= 0; --p)
		{
			double s = b[p];
			for(int q = p + 1; q < m; ++q) s -= S.U[m0 + p * m + q] * x[S.row[r0 + q]];
			x[S.row[r0 + p]] = s / S.U[m0 + p * m + p];
		}
	}
}

int PartnerOf(int a, int n, int bcLo, int bcHi)
{
	//  BoundaryCondition::ApplyEdge (BoundaryCondition.cpp:104-187):
	//  Symmetry mirrors the first two layers, Periodic copies the opposite side
	if(a < 2) return bcLo == YZ_BC_PERIODIC ? a + (n - 4) : 3 - a;
	if(a >= n - 2) return bcHi == YZ_BC_PERIODIC ? a - (n - 4) : 2 * (n - 2) - 1 - a;
	return a;
}

} // namespace

namespace {
inline double Bits(unsigned long long u) { double d; std::memcpy(&d, &u, sizeof d); return d; }

} // namespace

//==========================================================================
//  Step
//==========================================================================
Step::Step(int device, const yz_step_params &p, const double *h, const double *c, const double *s)
    : _device(device), _p(p)
{
	CheckParams(p);
	if(p.theta <= 0.0) throw UsageError("step: theta must be > 0 (the implicit scheme)");
	YZ_CUDA(cudaSetDevice(device));
	_solver.reset(new Solver(device));
	_st = _solver->Stream();
	YZ_CUDA(cudaEventCreate(&_e0)); YZ_CUDA(cudaEventCreate(&_e1));
	YZ_CUDA(cudaEventCreate(&_eA)); YZ_CUDA(cudaEventCreate(&_eB));
	const int nx = p.nx, ny = p.ny;
	_n = nx * ny;
	BuildPattern();
	BuildCoef();
	const size_t n = (size_t)_n;
	for(DBuf<double> *v : {&_h, &_c, &_s, &_hOld, &_hOld2, &_hNew, &_guess, &_axOld, &_axGuess, &_rhs, &_delta,
	                       &_evapOld, &_evapB})
	{
		v->reserve(n);
		YZ_CUDA(cudaMemsetAsync(v->get(), 0, n * sizeof(double), _st));
	}
	_ia.reserve((size_t)_nnz);
	YZ_CUDA(cudaMemsetAsync(_ia.get(), 0, (size_t)_nnz * sizeof(double), _st));
	_h.upload(h, n, _st); _c.upload(c, n, _st); _s.upload(s, n, _st);
	//  C_ImplicitSolver::SetX: phi_old = phi_old2 = phi_new = h
	YZ_CUDA(cudaMemcpyAsync(_hOld.get(), h, n * sizeof(double), cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_hOld2.get(), h, n * sizeof(double), cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_hNew.get(), h, n * sizeof(double), cudaMemcpyHostToDevice, _st));
	_red.reserve(8);
	//  the face properties (16 arrays of n, indexed by a face's low cell) and Pi
	_faceMem.reserve(19 * n);
	YZ_CUDA(cudaMemsetAsync(_faceMem.get(), 0, 19 * n * sizeof(double), _st));
	{
		double *m = _faceMem.get();
		double **slots[19] = {&_fb.x.vis, &_fb.x.sig, &_fb.x.FM, &_fb.x.DL, &_fb.x.fdLH, &_fb.x.fdHL, &_fb.x.gLH,
		                      &_fb.x.gHL, &_fb.y.vis, &_fb.y.sig, &_fb.y.FM, &_fb.y.DL, &_fb.y.fdLH, &_fb.y.fdHL,
		                      &_fb.y.gLH, &_fb.y.gHL, &_fb.piN, &_fb.phN, &_fb.dpN};
		for(int q = 0; q < 19; ++q) *slots[q] = m + (size_t)q * n;
	}
	_dt = p.dt; _dtOld = p.dt; _time = p.t_start;
	YZ_LAUNCH(KSetGhostRows, GridFor((long long)_nBcVal, 256), 256, 0, _st, _nBcVal, _dBcPos.get(),
	          _dBcVal.get(), (int)_ghost.size(), _dGhost.get(), _dBcRhs.get(), _ia.get(), _rhs.get());
	_cw.reserve(n);
	YZ_CUDA(cudaMemcpyAsync(_cw.get(), _c.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
	_conc = (p.conc_field != 0);
	if(_conc) BuildConc(c);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

Step::~Step()
{
	cudaSetDevice(_device);
	if(_st) cudaStreamSynchronize(_st);
	cudaEventDestroy(_e0); cudaEventDestroy(_e1); cudaEventDestroy(_eA); cudaEventDestroy(_eB);
}

//  The pattern the reference fixes in C_ImplicitSolver::Alloc
//  (ImplicitSolver.cpp:60-81): the ghost rows as BoundaryCondition2D::Apply
//  writes them (yz_bc.h), interior rows the capillary term's 13 points in
//  FullIdx order with the diagonal first.  ghost and partner: the ghost rows
//  and, where a ghost row copies one cell, that cell (else -1).
void BuildPattern2D(const yz_step_params &p, std::vector<int> &rowptr, std::vector<int> &col,
                    std::vector<int> &isbc, std::vector<int> &ghost, std::vector<int> &partner, BcPlan *planOut)
{
	const int nx = p.nx, ny = p.ny, n = nx * ny;
	BcPlan plan = BuildBcPlan(p);
	rowptr.assign((size_t)n + 1, 0);
	col.clear(); isbc.assign((size_t)n, 0);
	ghost = plan.ghost;
	partner = plan.partner;
	static const int off[13][2] = {{0, -2}, {-1, -1}, {0, -1}, {1, -1}, {-2, 0}, {-1, 0}, {0, 0}, {1, 0}, {2, 0},
	                               {-1, 1}, {0, 1}, {1, 1}, {0, 2}};
	size_t g = 0;
	for(int iy = 0; iy < ny; ++iy)
		for(int ix = 0; ix < nx; ++ix)
		{
			const int i = iy * nx + ix;
			const bool inside = ix >= 2 && ix < nx - 2 && iy >= 2 && iy < ny - 2;
			if(inside)
			{
				col.push_back(i);
				for(int q = 0; q < 13; ++q)
					if(q != oo) col.push_back((iy + off[q][1]) * nx + ix + off[q][0]);
			}
			else
			{
				isbc[(size_t)i] = 1;
				const std::vector<int> &c = plan.cols[g++];
				col.insert(col.end(), c.begin(), c.end());
			}
			rowptr[(size_t)i + 1] = (int)col.size();
		}
	if(planOut) *planOut = std::move(plan);
}

void CheckParams(const yz_step_params &p)
{
	if(p.nx < 8 || p.ny < 8) throw UsageError("step: the grid needs at least 4 x 4 cells");
	for(int e = 0; e < 4; ++e)
		if(p.bc[e] < YZ_BC_SYMMETRY || p.bc[e] > YZ_BC_OUTLET) throw UsageError("step: unknown edge kind");
	if((p.bc[0] == YZ_BC_PERIODIC) != (p.bc[1] == YZ_BC_PERIODIC) || (p.bc[2] == YZ_BC_PERIODIC) != (p.bc[3] == YZ_BC_PERIODIC))
		throw UsageError("step: a Periodic edge needs a Periodic opposite edge");
	if(!p.on_laplace) throw UsageError("step: the capillary term (Physics.LaplacePressure) must be enabled");
	if(p.conv_height < YZ_SCHEME_UPWIND1 || p.conv_height > YZ_SCHEME_VANLEER)
		throw UsageError("step: unknown Numerics.Convection.Height scheme");
	if(p.on_source && p.src_subregions < 1) throw UsageError("step: Physics.Source.SubRegions must be 1 or larger");
	if(p.conc_field != 0)
	{
		if(p.conv_conc < YZ_SCHEME_UPWIND1 || p.conv_conc > YZ_SCHEME_VANLEER)
			throw UsageError("step: unknown Numerics.Convection.Concentration scheme");
		if(!(p.theta_c > 0.0)) throw UsageError("step: theta_c must be > 0");
	}
}

void Step::BuildPattern()
{
	BuildPattern2D(_p, _rowptr, _col, _isbc, _ghost, _partner, &_bc);
	_nnz = (int)_col.size();
	//  the sorted mirror (CRS_Matrix::BuildSortPermutation, CRS_Matrix.cpp:360-384)
	std::vector<int> scol((size_t)_nnz), ssrc((size_t)_nnz);
	std::vector<std::pair<int, int>> tmp;
	for(int i = 0; i < _n; ++i)
	{
		const int st = _rowptr[(size_t)i], ed = _rowptr[(size_t)i + 1];
		tmp.clear();
		for(int q = st; q < ed; ++q) tmp.push_back({_col[(size_t)q], q});
		std::sort(tmp.begin(), tmp.end());
		for(int q = st; q < ed; ++q) { scol[(size_t)q] = tmp[(size_t)(q - st)].first; ssrc[(size_t)q] = tmp[(size_t)(q - st)].second; }
	}
	_solver->SetPattern(_n, _nnz, _rowptr.data(), scol.data(), ssrc.data());
	_dRowptr.upload(_rowptr.data(), _rowptr.size(), _st);
	std::vector<unsigned char> bc8(_isbc.begin(), _isbc.end());
	_dIsbc.upload(bc8.data(), bc8.size(), _st);
	_dGhost.upload(_ghost.data(), _ghost.size(), _st);
	_dPartner.upload(_partner.data(), _partner.size(), _st);
	//  the Newton matrix's ghost rows (their values in storage order) and
	//  right-hand side, and the SatisfyBCRows programme
	std::vector<int> pos;
	std::vector<double> val;
	for(size_t g = 0; g < _bc.ghost.size(); ++g)
		for(size_t k = 0; k < _bc.vals[g].size(); ++k)
		{
			pos.push_back(_rowptr[(size_t)_bc.ghost[g]] + (int)k);
			val.push_back(_bc.vals[g][k]);
		}
	_nBcVal = (int)pos.size();
	_dBcPos.upload(pos.data(), pos.size(), _st);
	_dBcVal.upload(val.data(), val.size(), _st);
	_dBcRhs.upload(_bc.rhs.data(), _bc.rhs.size(), _st);
	_dBc.Upload(_bc, _st);
}

//  The coefficient tables, computed as the reference's SetLinearCoef does
void Step::BuildCoef()
{
	Coef &k = _k;
	std::memset(&k, 0, sizeof k);
	const yz_step_params &p = _p;
	k.nx = p.nx; k.ny = p.ny;
	k.onL = p.on_laplace; k.onV = p.on_vgrav; k.onD = p.on_disjoining; k.onEvap = p.on_evap;
	k.theta = p.theta;
	const double dx = p.dx, dy = p.dy;
	const double dx2 = dx * dx, dy2 = dy * dy, dx4 = dx2 * dx2, dy4 = dy2 * dy2, dx2dy2 = dx2 * dy2;
	double (*C)[13] = k.cL;
	C[0][mm] = +1.0 / dx2dy2; C[0][om] = -1.0 / dx2dy2; C[0][Mo] = +1.0 / dx4;
	C[0][mo] = 1.0 * (-3.0 / dx4 - 2.0 / dx2dy2); C[0][oo] = 1.0 * (+3.0 / dx4 + 2.0 / dx2dy2);
	C[0][po] = -1.0 / dx4; C[0][mp] = +1.0 / dx2dy2; C[0][op] = -1.0 / dx2dy2;
	C[1][om] = -1.0 / dx2dy2; C[1][pm] = +1.0 / dx2dy2; C[1][mo] = -1.0 / dx4;
	C[1][oo] = 1.0 * (+3.0 / dx4 + 2.0 / dx2dy2); C[1][po] = 1.0 * (-3.0 / dx4 - 2.0 / dx2dy2);
	C[1][Po] = +1.0 / dx4; C[1][op] = -1.0 / dx2dy2; C[1][pp] = +1.0 / dx2dy2;
	C[2][oM] = +1.0 / dy4; C[2][mm] = +1.0 / dx2dy2; C[2][om] = 1.0 * (-3.0 / dy4 - 2.0 / dx2dy2);
	C[2][pm] = +1.0 / dx2dy2; C[2][mo] = -1.0 / dx2dy2; C[2][oo] = 1.0 * (+3.0 / dy4 + 2.0 / dx2dy2);
	C[2][po] = -1.0 / dx2dy2; C[2][op] = -1.0 / dy4;
	C[3][om] = -1.0 / dy4; C[3][mo] = -1.0 / dx2dy2; C[3][oo] = 1.0 * (+3.0 / dy4 + 2.0 / dx2dy2);
	C[3][po] = -1.0 / dx2dy2; C[3][mp] = +1.0 / dx2dy2; C[3][op] = 1.0 * (-3.0 / dy4 - 2.0 / dx2dy2);
	C[3][pp] = +1.0 / dx2dy2; C[3][oP] = +1.0 / dy4;
	static const int adj[4] = {mo, po, om, op};
	for(int d = 0; d < 4; ++d)
	{
		const double hs = (d / 2 == 0) ? dx : dy;
		const double h2 = hs * hs;
		k.cG[d][adj[d]] = +1.0 / h2;
		k.cG[d][oo] = -1.0 / h2;
	}
	k.coefL = 1.0 / 3.0;
	k.coefV = -1.0 * p.Bo / 3.0;
	k.coefD = p.Dp / 3.0;
	k.dx2 = dx2; k.dy2 = dy2; k.dx4 = dx4; k.dy4 = dy4; k.dx2dy2 = dx2dy2; k.dxx = dx; k.dyy = dy;
	k.hstar = p.hstar; k.pn = p.disj_n; k.pm = p.disj_m;
	k.slip = p.lambda_slip > 0;
	k.lam = p.lambda_slip > 0 ? p.lambda_slip : 0.0;
	k.a3 = 3.0 * k.lam;
	k.viscC0 = p.visc_c0; k.viscBase = p.visc_base; k.viscExp = p.visc_exp;
	k.sigC0 = p.sig_c0; k.sigBase = p.sig_base; k.sigCoef = p.sig_coef;
	k.Ev = p.Ev;
	k.evConc = p.ev_conc_func; k.evSpatial = p.ev_spatial; k.evHast = p.ev_hast_modify;
	k.evMr = p.ev_m_resin; k.evMs = p.ev_m_solvent; k.evPowN = p.ev_power_n; k.evConcR = p.ev_conc_r;
	k.evNegExp = p.ev_negpow_exp; k.evNegRmax = p.ev_negpow_rmax; k.evHast_h = p.ev_h_ast;
	k.evDr = dx < dy ? dx : dy;
	k.xmin = p.xmin; k.ymin = p.ymin; k.dx = dx; k.dy = dy; k.dx2h = dx * 0.5; k.dy2h = dy * 0.5;
	//  the upwinded terms
	k.onPG = p.on_pgrav; k.onSC = p.on_marangoni; k.onCF = p.on_centrifugal;
	for(int e = 0; e < 4; ++e)
	{
		k.wall[e] = (p.bc[e] == YZ_BC_SYMMETRY || p.bc[e] == YZ_BC_PINNING);   // BoundaryCondition::IsWall
		k.pinned[e] = (p.bc[e] == YZ_BC_PINNING);
	}
	k.hI = MakeInterp(p.conv_height);
	const double pg[2] = {p.Pgx, p.Pgy};
	for(int a = 0; a < 2; ++a) { k.pgMag[a] = pg[a] / 3.0; k.pgSign[a] = pg[a] >= 0 ? 1.0 : -1.0; }
	k.cfMag = p.Sp / 3.0;
	k.cnt[0] = p.rot_x; k.cnt[1] = p.rot_y;
	k.scMag = p.As * p.Ma / 2.0;
	//  the concentration equation
	ConcCoef &q = _kc;
	std::memset(&q, 0, sizeof q);
	q.nx = p.nx; q.ny = p.ny;
	q.conv = p.conc_convection; q.diff = p.conc_diffusion;
	q.th = p.theta_c;
	q.Df = p.Df; q.dC0 = p.diff_c0; q.dBase = p.diff_base; q.dExp = p.diff_exp;
	q.dxx = dx; q.dyy = dy;
	q.cI = MakeInterp(p.conv_conc);
}

double Step::ReadMax(int slot)
{
	unsigned long long u = 0;
	YZ_CUDA(cudaMemcpyAsync(&u, _red.get() + slot, sizeof(u), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	return Bits(u);
}

void Step::ZeroMax(int slot) { YZ_CUDA(cudaMemsetAsync(_red.get() + slot, 0, sizeof(unsigned long long), _st)); }

//  the face properties of the film (H, C) into _fb (with the Jacobian's
//  derivatives when J), and Pi of every cell
void Step::FaceProps(const double *H, const double *C, bool J)
{
	const int nF = (_p.nx - 3) * (_p.ny - 4) + (_p.nx - 4) * (_p.ny - 3);
	if(J) YZ_LAUNCH(KFaceProps<true>, GridFor(nF, 128, 148 * 32), 128, 0, _st, _k, H, C, _fb);
	else YZ_LAUNCH(KFaceProps<false>, GridFor(nF, 128, 148 * 32), 128, 0, _st, _k, H, C, _fb);
	if(_k.onD) YZ_LAUNCH(KCellPi, GridFor(_n, 256), 256, 0, _st, _k, _n, H, _fb);
}

void Step::Assemble(int mode, const double *hField, const double *cField, double dt)
{
	//  one fused pass: the reference's h.assemble, h.jacobian and h.rhs
	YZ_PROF("h.assemble", _st);
	FaceProps(hField, cField, mode == 1);
	UpBuf up;
	up.base = nullptr; up.stride = _n;
	if(_k.onPG || _k.onCF || _k.onSC)
	{
		_upMem.reserve((size_t)48 * _n);
		up.base = _upMem.get();
		const dim3 grid(GridFor(_n, 128, 148 * 16), 6);
		if(mode == 1) YZ_LAUNCH(KUpwindFaces<true>, grid, 128, 0, _st, _k, hField, cField, _fb, up);
		else YZ_LAUNCH(KUpwindFaces<false>, grid, 128, 0, _st, _k, hField, cField, _fb, up);
	}
	RowOut o;
	o.ia = _ia.get(); o.ax = mode == 0 ? _axOld.get() : _axGuess.get();
	o.evapOld = _evapOld.get(); o.evapB = _evapB.get(); o.rhs = _rhs.get();
	o.hOld = _hOld.get(); o.axOld = _axOld.get(); o.rhsMax = _red.get() + kSlotRhs;
	o.src = _p.on_source ? _src.get() : nullptr;
	const int nIn = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KAssemble, GridFor(nIn, 128, 148 * 32), 128, 0, _st, _k, mode, dt, _dRowptr.get(), hField, cField,
	          _s.get(), o, _fb, up);
}

//  the ghost rows of x satisfied exactly (SatisfyBCRows with the Newton
//  system's right-hand side on them)
void Step::SatisfyGhosts(double *x)
{
	if(_bc.simple)
	{
		YZ_LAUNCH(KGhostCopy, GridFor((long long)_ghost.size(), 256), 256, 0, _st, (int)_ghost.size(), _dGhost.get(),
		          _dPartner.get(), x);
		return;
	}
	YZ_LAUNCH(KSatisfyBC, GridFor((long long)_dBc.nSets, 128), 128, 0, _st, _dBc.Sets(nullptr), x);
}

void Step::SatisfyConcGhosts(double *x, const double *rhsVec)
{
	if(_bcC.simple)
	{
		//  every ghost copies one cell: with the equation's right-hand side
		//  (zero) the copy; the d system's is done by KConcUpdate
		YZ_LAUNCH(KGhostCopy, GridFor((long long)_ghost.size(), 256), 256, 0, _st, (int)_ghost.size(), _dGhost.get(),
		          _dPartner.get(), x);
		return;
	}
	YZ_LAUNCH(KSatisfyBC, GridFor((long long)_dBcC.nSets, 128), 128, 0, _st, _dBcC.Sets(rhsVec), x);
}

//  The nozzle at the middle of the step (SourceBase::SetEvalTime in
//  BeforeNKLoop, HeightEquationBase.h:1339): its position on the arm
//  (SourceBase::NozzlePos: the arm's angle is the start angle plus the rate
//  times the integral of a trapezoid ramp) and the flow rate
//  (FlowRateNow: 1 - exp(-t / tau) of the rate), then every cell's supply
void Step::UpdateSource(double dt)
{
	const yz_step_params &p = _p;
	const double tt = _time + 0.5 * dt;
	const double Ts = p.src_ramp, Tm = p.src_plateau;
	const double t = std::max(0.0, tt - p.src_t0);
	double swept;
	if(t <= Ts) swept = (Ts > 0) ? 0.5 * t * t / Ts : 0.0;
	else if(t <= Ts + Tm) swept = 0.5 * Ts + (t - Ts);
	else if(t <= 2.0 * Ts + Tm)
	{
		const double tau = t - Ts - Tm;
		swept = 0.5 * Ts + Tm + tau - 0.5 * tau * tau / Ts;
	}
	else swept = Ts + Tm;
	const double theta = p.src_angle0 + p.src_omega * swept;
	const double xn = p.src_arm_x + p.src_arm * std::cos(theta);
	const double yn = p.src_arm_y + p.src_arm * std::sin(theta);
	double coef = 1.0;
	if(!(std::fabs(p.src_tau) <= std::numeric_limits<double>::epsilon())) coef = 1.0 - std::exp(-tt / p.src_tau);
	const double flow = p.src_rate * coef;
	_src.reserve((size_t)_n);
	YZ_LAUNCH(KSource, GridFor(_n, 256), 256, 0, _st, _k, xn, yn, p.src_radius, p.src_subregions, flow, _src.get());
}

//  one Newton-Kantorovich attempt at the present dt (NKLoop)
bool Step::NKLoop(int &iter, double &resid, yz_step_stats &stats)
{
	const int n = _n, g = GridFor(n, 256);
	const double dt = _dt;
	_nkIter = 0;
	YZ_CUDA(cudaMemcpyAsync(_guess.get(), _hOld.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
	//  opt extrap
	_extrapMove = 0;
	if(_p.on_source) UpdateSource(dt);
	if(!_extrapBlocked)
	{
		const double r = (_dtOld > 0) ? dt / _dtOld : 0.0;
		if(r > 0)
		{
			ZeroMax(kSlotMove);
			int *bad = reinterpret_cast<int *>(_red.get() + kSlotBad);
			YZ_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), _st));
			YZ_LAUNCH(KExtrapCheck, g, 256, 0, _st, n, _hOld.get(), _hOld2.get(), _dIsbc.get(), r, bad, _red.get() + kSlotMove);
			const double move = ReadMax(kSlotMove);
			int hbad = 0;
			YZ_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, _st));
			YZ_CUDA(cudaStreamSynchronize(_st));
			if(!hbad && move > 0)
			{
				YZ_LAUNCH(KExtrapApply, g, 256, 0, _st, n, _hOld.get(), _hOld2.get(), r, _guess.get());
				_extrapMove = move;
			}
		}
	}
	//  BeforeNKLoop (HeightEquationBase.h:1314-1387): the working field is the
	//  committed one; with the concentration, the limiter and the reference
	//  of the coupled correction at the step's start, the face fluxes there
	//  (F0) and the solves of the step from d = 0.  Then SetMatrixA and
	//  A(h^n) h^n with evapOld at h^n.
	_coupled = 0;
	YZ_CUDA(cudaMemcpyAsync(_cw.get(), _c.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
	if(_conc)
	{
		YZ_CUDA(cudaMemcpyAsync(_cLim.get(), _c.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
		YZ_CUDA(cudaMemcpyAsync(_cPrev.get(), _c.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
		FaceFluxes(_h.get(), _c.get(), _F0x.get(), _F0y.get(), dt, false);
		YZ_CUDA(cudaMemsetAsync(_dC.get(), 0, (size_t)n * sizeof(double), _st));
	}
	Assemble(0, _hOld.get(), _c.get(), dt);

	double residEqOld = 1e40, residFirst = 0, residBest = 1e40;
	int stall = 0;
	const int stallLimit = 5;
	bool done = false;
	int outer;
	for(outer = 0; outer < _p.nk_max; ++outer)
	{
		//  EveryNKLoop: the working field's h is phi_guess; with the
		//  concentration, its solve at this film first (a failed one fails
		//  the pass and with it the attempt).  Solve(): assembly at the film
		//  and the working field's c.
		if(_conc)
		{
			YZ_PROF("h.couple", _st);
			if(!ConcPass(dt, stats)) { done = false; break; }
		}
		ZeroMax(kSlotRhs);
		YZ_CUDA(cudaEventRecord(_e0, _st));
		Assemble(1, _guess.get(), _cw.get(), dt);
		YZ_CUDA(cudaEventRecord(_e1, _st));
		++_nkIter;
		//  opt ew (NewtonKantorovich.cpp:108-126)
		double eps = _p.lin.epsilon;
		{
			const double kEtaMax = 1.0e-4;
			const double rn = ReadMax(kSlotRhs);
			float ams = 0; YZ_CUDA(cudaEventElapsedTime(&ams, _e0, _e1)); stats.assemble_ms += ams;
			double eta = kEtaMax;
			if(_nkIter > 1 && _ewRhsPrev > 0)
			{
				const double ratio = rn / _ewRhsPrev;
				eta = 0.9 * ratio * ratio;
				const double safe = 0.9 * _ewEta * _ewEta;
				if(safe > 0.1 && safe > eta) eta = safe;
			}
			if(eta > kEtaMax) eta = kEtaMax;
			if(eta < _p.lin.epsilon) eta = _p.lin.epsilon;
			_ewEta = eta;
			_ewRhsPrev = rn;
			eps = eta;
		}
		yz_settings ls = _p.lin;
		ls.epsilon = eps;
		ls.conc = 0;
		int it = 0; double res = 0;
		//  the learned preconditioner reads the pass's film as a feature, and
		//  is trained once the solves that collect its pairs are done
		if(_learned)
		{
			_solver->SetAux(_guess.get());
			if(!_learned->Trained() && _solver->CollectLeft() == 0) TrainLearned(stats);
		}
		const int r0 = _solver->Rebuilds();
		int ch;
		{
			YZ_PROF("h.linsolve", _st);
			ch = _solver->Solve(ls, _ia.get(), _rhs.get(), _delta.get(), it, res);
		}
		double su = 0, sit = 0; _solver->Timing(&su, &sit);
		stats.setup_ms += su; stats.solve_ms += sit;
		stats.amg_setups += _solver->Rebuilds() - r0;
		stats.linear_iterations += it;
		ZeroMax(kSlotDelta);
		if(ch == 0) SatisfyGhosts(_delta.get());
		else YZ_CUDA(cudaMemsetAsync(_delta.get(), 0, (size_t)n * sizeof(double), _st));
		YZ_LAUNCH(KAbsMax, g, 256, 0, _st, n, _delta.get(), _red.get() + kSlotDelta);
		double residEq = ReadMax(kSlotDelta);
		//  the convergence test takes the larger of the film's correction and
		//  the concentration's (NewtonKantorovich.cpp:323)
		if(_coupled > residEq) residEq = _coupled;
		_lastResid = residEq;
		if(ch != 0) { done = false; break; }
		if(outer == 0) residFirst = residEq;
		if(residEq < residBest * 0.9) { residBest = residEq; stall = 0; }
		else ++stall;
		if(stall > stallLimit)
		{
			ZeroMax(kSlotPhi);
			YZ_LAUNCH(KAbsMax, g, 256, 0, _st, n, _guess.get(), _red.get() + kSlotPhi);
			const double floorPhi = 1000.0 * std::numeric_limits<double>::epsilon() * ReadMax(kSlotPhi);
			const bool solved = (residEq < _p.nk_eps) || (residFirst > 0 && residEq < residFirst * 1.0e-4) || (residEq <= floorPhi);
			done = solved;
			break;
		}
		const double alpha = (residEq > residEqOld) ? 0.5 : 1.0;
		YZ_LAUNCH(KAxpyAlpha, g, 256, 0, _st, n, _delta.get(), alpha, _guess.get());
		if(outer >= _p.nk_min - 1)
		{
			if(residEq < _p.nk_eps) { done = true; break; }
			if(_p.nk_eps_rel > 0 && residFirst > 0 && residEq < residFirst * _p.nk_eps_rel) { done = true; break; }
		}
		residEqOld = residEq;
	}
	iter = outer + 1;
	resid = _lastResid;
	return done;
}

//  TimeAdvance (NewtonKantorovich.cpp:424-486) and the clock (TimeSteps.cpp:121-160)
void Step::SetLearned(const yz_learned_cfg *cfg)
{
	YZ_CUDA(cudaSetDevice(_device));
	if(!cfg)
	{
		_solver->SetLearned(nullptr, 0, 0, 0, 1.0);
		_learned.reset();
		return;
	}
	if(cfg->collect_solves < 1 || cfg->samples_per_solve < 1 || cfg->capacity < 2 || cfg->train_iters < 0 ||
	   cfg->batch < 1 || !(cfg->lr > 0) || cfg->holdout < 0 || !(cfg->cap_factor > 0) ||
	   (cfg->activation != 0 && cfg->activation != 1))
		throw UsageError("set_learned: collect_solves, samples_per_solve, batch >= 1, capacity >= 2, lr and "
		                 "cap_factor > 0, train_iters and holdout >= 0");
	_lcfg = *cfg;
	_solver->SetLearned(nullptr, 0, 0, 0, 1.0);
	_learned.reset(new Learned(_device, _p.nx, _p.ny, cfg->capacity, cfg->seed, cfg->activation));
	_solver->SetLearned(_learned.get(), 1, cfg->collect_solves, cfg->samples_per_solve, cfg->cap_factor);
	_lValErr = -1.0;
	_lLoss = -1.0;
}

//  Adam on the pairs the film's solves collected; then the film's solves try
//  the network first
void Step::TrainLearned(yz_step_stats &stats)
{
	cudaEvent_t e0, e1;
	YZ_CUDA(cudaEventCreate(&e0));
	YZ_CUDA(cudaEventCreate(&e1));
	YZ_CUDA(cudaEventRecord(e0, _st));
	const int hold = std::min(_lcfg.holdout, std::max(0, _learned->Samples() - 1));
	double val = -1.0;
	_lLoss = _learned->Train(_lcfg.train_iters, _lcfg.batch, _lcfg.lr, hold, &val, _st);
	_lValErr = val;
	YZ_CUDA(cudaEventRecord(e1, _st));
	YZ_CUDA(cudaEventSynchronize(e1));
	float ms = 0;
	YZ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	stats.learned_train_ms += ms;
	_solver->SetLearned(_learned.get(), 2, 0, 0, _lcfg.cap_factor);
}

void Step::Advance(int nsteps, yz_step_stats &stats)
{
	YZ_CUDA(cudaSetDevice(_device));
	const size_t bytes = (size_t)_n * sizeof(double);
	const int g = GridFor(_n, 256);
	const long long l0 = t_launches;
	const Solver::LearnedStats ls0 = _solver->LStats();
	YZ_CUDA(cudaEventRecord(_eA, _st));
	for(int step = 0; step < nsteps; ++step)
	{
		YZ_PROF("step", _st);
		YZ_CUDA(cudaMemcpyAsync(_hOld2.get(), _hOld.get(), bytes, cudaMemcpyDeviceToDevice, _st));
		YZ_CUDA(cudaMemcpyAsync(_hOld.get(), _hNew.get(), bytes, cudaMemcpyDeviceToDevice, _st));
		bool timeStepDone = false;
		int iter = 0;
		double resid = 0;
		do
		{
			bool ch = NKLoop(iter, resid, stats);
			stats.newton_iterations += iter;
			if(!ch && _extrapMove > 0)
			{
				_extrapBlocked = true;
				ch = NKLoop(iter, resid, stats);
				stats.newton_iterations += iter;
				_extrapBlocked = false;
			}
			if(_p.dt_control)
			{
				double criterion = -1;
				if(ch)
				{
					//  LocalTruncationCriterion(phi_guess)
					double th = _p.dt_criterion;
					if(std::fabs(th) <= std::numeric_limits<double>::min()) th = 1.0e-2;
					if(std::fabs(_dtOld) <= std::numeric_limits<double>::min()) criterion = 1.0;
					else
					{
						ZeroMax(kSlotPhi);
						YZ_LAUNCH(KAbsMax, g, 256, 0, _st, _n, _hOld.get(), _red.get() + kSlotPhi);
						const double wfloor = _p.dt_scale_floor * ReadMax(kSlotPhi);
						ZeroMax(kSlotLte);
						YZ_LAUNCH(KLte, g, 256, 0, _st, _n, _guess.get(), _hOld.get(), _hOld2.get(), _dtOld, _dt, wfloor,
						          _red.get() + kSlotLte);
						criterion = 1.0 - ReadMax(kSlotLte) / th;
					}
				}
				//  TimeStepAdjustment (ImplicitSolver.cpp:144-190)
				double dtNext = _dt;
				if(criterion > 0.0)
				{
					timeStepDone = true;
					if(criterion > 0.90 && dtNext < _p.dt_max)
					{
						if(++_adjustCount >= _p.dt_keep_steps)
						{
							_adjustCount = 0;
							dtNext /= _p.dt_change_factor;
							if(dtNext > _p.dt_max) dtNext = _p.dt_max;
							if(!(dtNext < _p.dt_min || _p.dt_max < dtNext)) _pendingDt = dtNext;
						}
					}
				}
				else
				{
					dtNext *= _p.dt_change_factor;
					if(dtNext < _p.dt_min)
						throw StepFailed("TimeStepAdjustment(). Under flow: the requested step fell below "
						                 "Numerics.TimeStepControl.MinDt.");
					if(!(dtNext < _p.dt_min || _p.dt_max < dtNext)) _dt = dtNext;
					++stats.retries;
				}
			}
			else
			{
				if(!ch)
					throw StepFailed("Newton-Kantorovich: the step did not converge at the fixed step, and with "
					                 "Numerics.TimeStepControl.Enable = false it cannot be retried at a shorter "
					                 "one. Shorten Numerics.InitialDt or enable the time-step control.");
				timeStepDone = true;
			}
		} while(!timeStepDone);
		YZ_CUDA(cudaMemcpyAsync(_hNew.get(), _guess.get(), bytes, cudaMemcpyDeviceToDevice, _st));
		//  AfterNKLoop: with the concentration, the step of h c completed
		//  (ConcCommit); the field takes the film
		if(_conc)
		{
			YZ_PROF("h.after", _st);
			ConcCommit(_dt, stats);
		}
		YZ_CUDA(cudaMemcpyAsync(_h.get(), _guess.get(), bytes, cudaMemcpyDeviceToDevice, _st));
		//  the energy budget of the film the step reached, the energy
		//  dissipated over the step at its Crank-Nicolson weighting, and
		//  the balance (WellMixedModelBase.h:1405-1411)
		if(_energyOn)
		{
			const double f0 = _enF, d0 = _enD;
			Energy(_enF, _enD);
			_enDiss += 0.5 * (d0 + _enD) * _dt;
			_enBal = (_enF - f0) / _dt + 0.5 * (d0 + _enD);
		}
		//  the clock: ++ (TimeSteps.cpp:121-160)
		_time += _dt;
		_dtOld = _dt;
		if(_pendingDt > 0) { _dt = _pendingDt; _pendingDt = 0; }
		stats.steps += 1;
		stats.last_resid = resid;
	}
	stats.time = _time;
	stats.dt = _dt;
	{
		const Solver::LearnedStats &ls1 = _solver->LStats();
		stats.learned_solves += ls1.solves - ls0.solves;
		stats.learned_fallbacks += ls1.fallbacks - ls0.fallbacks;
		stats.learned_iterations += ls1.iterations - ls0.iterations;
		stats.learned_samples = _learned ? _learned->Samples() : 0;
		stats.learned_val_err = _lValErr;
		stats.learned_loss = _lLoss;
	}
	if(_energyOn)
	{
		stats.energy_F = _enF; stats.energy_D = _enD;
		stats.energy_dissipated = _enDiss; stats.energy_balance = _enBal;
	}
	YZ_CUDA(cudaEventRecord(_eB, _st));
	YZ_CUDA(cudaEventSynchronize(_eB));
	float ms = 0;
	YZ_CUDA(cudaEventElapsedTime(&ms, _eA, _eB));
	stats.device_ms = ms;
	stats.launches = t_launches - l0;
}

void Step::SetFields(const double *h, const double *c)
{
	YZ_CUDA(cudaSetDevice(_device));
	const size_t bytes = (size_t)_n * sizeof(double);
	if(h)
	{
		YZ_CUDA(cudaMemcpyAsync(_h.get(), h, bytes, cudaMemcpyHostToDevice, _st));
		YZ_CUDA(cudaMemcpyAsync(_hNew.get(), _h.get(), bytes, cudaMemcpyDeviceToDevice, _st));
	}
	if(c)
	{
		YZ_CUDA(cudaMemcpyAsync(_c.get(), c, bytes, cudaMemcpyHostToDevice, _st));
		YZ_CUDA(cudaMemcpyAsync(_cw.get(), _c.get(), bytes, cudaMemcpyDeviceToDevice, _st));
		//  C_ImplicitSolver::SetX of the concentration equation
		if(_conc) YZ_CUDA(cudaMemcpyAsync(_c0.get(), _c.get(), bytes, cudaMemcpyDeviceToDevice, _st));
	}
}

//  The state of the step between two calls, the counterpart of the
//  reference's RestartState (IO/RestartState.h:57): the committed film and
//  concentration, the films of the two steps before (phi_old, phi_old2) and
//  the last accepted one (phi_new), the last Newton correction (the next
//  solve's initial guess, LastCorrection), the clock and its controller
//  (dt, dt of the step before, a pending dt change, the step-keep count),
//  the Eisenstat-Walker and extrapolation memory, the solvers' TryBackoff
//  counters and the energy history.  Layout: kStateHead doubles -- a tag,
//  n, then the scalars in the order written below -- then six fields of n.
namespace { constexpr size_t kStateHead = 24; constexpr double kStateTag = 20261204.0; }

size_t Step::StateSize() const { return kStateHead + (size_t)6 * _n; }

void Step::GetState(double *out)
{
	YZ_CUDA(cudaSetDevice(_device));
	const size_t n = (size_t)_n;
	double *o = out;
	std::fill(o, o + kStateHead, 0.0);
	o[0] = kStateTag; o[1] = (double)_n;
	o[2] = _dt; o[3] = _dtOld; o[4] = _time; o[5] = _pendingDt; o[6] = (double)_adjustCount;
	o[7] = (double)_nkIter; o[8] = _ewEta; o[9] = _ewRhsPrev; o[10] = _extrapMove; o[11] = _lastResid;
	o[12] = _energyOn ? 1.0 : 0.0; o[13] = _enF; o[14] = _enD; o[15] = _enDiss; o[16] = _enBal;
	const std::vector<double> mh = _solver->Memory();
	o[17] = mh.size() > 0 ? mh[0] : 0.0; o[18] = mh.size() > 1 ? mh[1] : 0.0;
	if(_solverC)
	{
		const std::vector<double> mc = _solverC->Memory();
		o[19] = mc.size() > 0 ? mc[0] : 0.0; o[20] = mc.size() > 1 ? mc[1] : 0.0;
	}
	double *f = out + kStateHead;
	const DBuf<double> *fields[6] = {&_h, &_c, &_hOld, &_hOld2, &_hNew, &_delta};
	for(int k = 0; k < 6; ++k) fields[k]->download(f + (size_t)k * n, n, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

void Step::SetState(const double *in, size_t len)
{
	YZ_CUDA(cudaSetDevice(_device));
	if(len != StateSize() || in[0] != kStateTag || in[1] != (double)_n)
		throw UsageError("set_state: not a state of this step (wrong size or grid)");
	const size_t n = (size_t)_n;
	_dt = in[2]; _dtOld = in[3]; _time = in[4]; _pendingDt = in[5]; _adjustCount = (int)in[6];
	_nkIter = (int)in[7]; _ewEta = in[8]; _ewRhsPrev = in[9]; _extrapMove = in[10]; _lastResid = in[11];
	_energyOn = in[12] != 0.0; _enF = in[13]; _enD = in[14]; _enDiss = in[15]; _enBal = in[16];
	_solver->SetMemory(in + 17, 2);
	if(_solverC) _solverC->SetMemory(in + 19, 2);
	const double *f = in + kStateHead;
	DBuf<double> *fields[6] = {&_h, &_c, &_hOld, &_hOld2, &_hNew, &_delta};
	for(int k = 0; k < 6; ++k) fields[k]->upload(f + (size_t)k * n, n, _st);
	YZ_CUDA(cudaMemcpyAsync(_cw.get(), _c.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
	if(_conc) YZ_CUDA(cudaMemcpyAsync(_c0.get(), _c.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
}

void Step::Energy(double &F, double &D)
{
	YZ_CUDA(cudaSetDevice(_device));
	const int nIn = (_p.nx - 4) * (_p.ny - 4);
	_enFx.reserve((size_t)_n); _enFy.reserve((size_t)_n); _enOut.reserve(2);
	//  FaceFluxes' film flag and the reduction scratch, which the
	//  concentration equation holds when it is on
	_iflags.reserve(4);
	_partStep.reserve((size_t)2 * RedBlocks(_n));
	if(_cntStep.get() == nullptr)
	{
		_cntStep.reserve(4);
		YZ_CUDA(cudaMemsetAsync(_cntStep.get(), 0, 4 * sizeof(unsigned int), _st));
	}
	FaceFluxes(_h.get(), _c.get(), _enFx.get(), _enFy.get(), 0.0, false);
	EnergyPar e;
	e.bo = _p.Bo; e.dp = _p.Dp; e.hstar = _p.hstar; e.pn = _p.disj_n; e.pm = _p.disj_m;
	e.capillary = _p.on_laplace ? 1 : 0;
	e.perX = _p.bc[0] == YZ_BC_PERIODIC ? 1 : 0;
	e.perY = _p.bc[2] == YZ_BC_PERIODIC ? 1 : 0;
	YZ_LAUNCH(KEnergy, RedBlocks(nIn), kRT, 0, _st, _k, e, _h.get(), _c.get(), _s.get(), _enFx.get(), _enFy.get(),
	          StepRed(2), _enOut.get());
	double out[2];
	YZ_CUDA(cudaMemcpyAsync(out, _enOut.get(), sizeof out, cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	F = out[0];
	D = out[1];
}

void Step::SetEnergy(bool on)
{
	_energyOn = on;
	_enDiss = 0; _enBal = 0;
	if(on) Energy(_enF, _enD);
}

void Step::GetFields(double *h, double *c)
{
	YZ_CUDA(cudaSetDevice(_device));
	if(h) _h.download(h, (size_t)_n, _st);
	if(c) _c.download(c, (size_t)_n, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

int Step::Pattern(int *rowptr, int *col, int *bc) const
{
	if(rowptr) std::copy(_rowptr.begin(), _rowptr.end(), rowptr);
	if(col) std::copy(_col.begin(), _col.end(), col);
	if(bc) for(int i = 0; i < _n; ++i) bc[i] = _isbc[(size_t)i];
	return _nnz;
}

void Step::System(const double *hOld, const double *h, double dt, double *ia, double *rhs)
{
	YZ_CUDA(cudaSetDevice(_device));
	const size_t bytes = (size_t)_n * sizeof(double);
	YZ_CUDA(cudaMemcpyAsync(_hOld.get(), hOld, bytes, cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_guess.get(), h, bytes, cudaMemcpyHostToDevice, _st));
	if(_p.on_source) UpdateSource(dt);
	Assemble(0, _hOld.get(), _c.get(), dt);
	ZeroMax(kSlotRhs);
	Assemble(1, _guess.get(), _c.get(), dt);
	_ia.download(ia, (size_t)_nnz, _st);
	_rhs.download(rhs, (size_t)_n, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

//==========================================================================
//  The well-mixed concentration equation
//==========================================================================
//  Its pattern (C_ImplicitSolver::Alloc with ConcEquationBase::SetMatrixA,
//  ConcEquationBase.h:243-259): the boundary rows of BoundaryCondition2D::
//  Apply for the concentration (EqualVal [diag, partner] on Symmetry and
//  Periodic edges, as for the film), interior rows the diagonal and the wide
//  set in WideIdx order.
void BuildConcPattern2D(const yz_step_params &p, std::vector<int> &rowptr, std::vector<int> &col, const BcPlan &plan)
{
	const int nx = p.nx, ny = p.ny, n = nx * ny;
	rowptr.assign((size_t)n + 1, 0);
	col.clear();
	static const int wide[8][2] = {{0, -2}, {0, -1}, {-2, 0}, {-1, 0}, {1, 0}, {2, 0}, {0, 1}, {0, 2}};
	size_t g = 0;
	for(int iy = 0; iy < ny; ++iy)
		for(int ix = 0; ix < nx; ++ix)
		{
			const int i = iy * nx + ix;
			col.push_back(i);
			const bool inside = ix >= 2 && ix < nx - 2 && iy >= 2 && iy < ny - 2;
			if(inside)
				for(int q = 0; q < 8; ++q) col.push_back((iy + wide[q][1]) * nx + ix + wide[q][0]);
			else
			{
				//  the ghost row as BoundaryCondition2D::Apply writes the
				//  concentration's (its diagonal is the one pushed above)
				const std::vector<int> &c = plan.cols[g++];
				col.insert(col.end(), c.begin() + 1, c.end());
			}
			rowptr[(size_t)i + 1] = (int)col.size();
		}
}

void Step::BuildConc(const double *cHost)
{
	const size_t n = (size_t)_n;
	_bcC = BuildBcPlan(_p, kBcFieldConc, cHost);
	BuildConcPattern2D(_p, _rowptrC, _colC, _bcC);
	_nnzC = (int)_colC.size();
	std::vector<int> scol((size_t)_nnzC), ssrc((size_t)_nnzC);
	std::vector<std::pair<int, int>> tmp;
	for(int i = 0; i < _n; ++i)
	{
		const int st = _rowptrC[(size_t)i], ed = _rowptrC[(size_t)i + 1];
		tmp.clear();
		for(int q = st; q < ed; ++q) tmp.push_back({_colC[(size_t)q], q});
		std::sort(tmp.begin(), tmp.end());
		for(int q = st; q < ed; ++q) { scol[(size_t)q] = tmp[(size_t)(q - st)].first; ssrc[(size_t)q] = tmp[(size_t)(q - st)].second; }
	}
	_solverC.reset(new Solver(_device, _st));
	_solverC->SetPrecision(_precision);
	_solverC->SetAmgReuse(_amgReuse);
	_solverC->SetGraphLoop(_graphLoop);
	_solverC->SetPattern(_n, _nnzC, _rowptrC.data(), scol.data(), ssrc.data());
	_dRowptrC.upload(_rowptrC.data(), _rowptrC.size(), _st);
	std::vector<int> pall(n);
	for(int i = 0; i < _n; ++i) pall[(size_t)i] = i;
	for(size_t g = 0; g < _ghost.size(); ++g)
		if(_partner[g] >= 0) pall[(size_t)_ghost[g]] = _partner[g];
	_dPartnerAll.upload(pall.data(), n, _st);
	for(DBuf<double> *v : {&_c0, &_cLim, &_cPrev, &_cx, &_cxLast, &_dC, &_rhsC, &_F0x, &_F0y, &_F1x, &_F1y, &_evpStep,
	                       &_rho, &_room, &_give, &_cPre, &_G2x, &_G2y})
	{
		v->reserve(n);
		YZ_CUDA(cudaMemsetAsync(v->get(), 0, n * sizeof(double), _st));
	}
	for(DBuf<double> *v : {&_rowSum, &_accY})
	{
		v->reserve((size_t)_p.ny);
		YZ_CUDA(cudaMemsetAsync(v->get(), 0, (size_t)_p.ny * sizeof(double), _st));
	}
	_sums.reserve(4);
	_partStep.reserve((size_t)2 * RedBlocks(_n));
	_cntStep.reserve(4);
	YZ_CUDA(cudaMemsetAsync(_cntStep.get(), 0, 4 * sizeof(unsigned int), _st));
	_iflags.reserve(4);
	//  the matrix: the boundary rows once (the concentration's, yz_bc.h),
	//  the interior rows every solve
	std::vector<double> vals((size_t)_nnzC, 0.0);
	for(size_t g = 0; g < _bcC.ghost.size(); ++g)
	{
		const int i = _bcC.ghost[g];
		for(size_t k = 0; k < _bcC.vals[g].size(); ++k) vals[(size_t)_rowptrC[(size_t)i] + k] = _bcC.vals[g][k];
	}
	_iaC.upload(vals.data(), vals.size(), _st);
	//  the copy form of the ghosts reads the film's ghost and partner lists:
	//  only where the two plans copy alike
	_bcC.simple = _bcC.simple && _bc.simple && _bcC.ghost == _bc.ghost && _bcC.partner == _bc.partner;
	_dBcC.Upload(_bcC, _st);
	_dBcCRhs.upload(_bcC.rhs.data(), _bcC.rhs.size(), _st);
	_dColC.upload(_colC.data(), _colC.size(), _st);
	//  C_ImplicitSolver::SetX: c0 = c
	YZ_CUDA(cudaMemcpyAsync(_c0.get(), _c.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
}

RedScratch Step::StepRed(int site)
{
	RedScratch r;
	r.part = _partStep.get();
	r.counter = _cntStep.get() + site;
	r.maxBlocks = RedBlocks(_n);
	return r;
}

//  FaceVolumeFluxes of the film (H, C) into Fx / Fy; with withEvap, the
//  evaporation of the step (StepSources); returns FilmNotPositive
int Step::FaceFluxes(const double *H, const double *C, double *Fx, double *Fy, double dt, bool withEvap)
{
	const int nIn = (_p.nx - 4) * (_p.ny - 4);
	int *bad = _iflags.get();
	YZ_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), _st));
	FaceProps(H, C, false);
	YZ_LAUNCH(KFaceFlux, dim3(GridFor(nIn, 128, 148 * 16), 2), 128, 0, _st, _k, H, C, _s.get(), Fx, Fy, _evapOld.get(), dt,
	          withEvap ? _evpStep.get() : nullptr, bad, _fb);
	int h = 0;
	YZ_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	return h;
}

void Step::ConcInputs(ConcIn &in) const
{
	in.c0 = _c0.get(); in.cLim = _cLim.get(); in.h0 = _hOld.get(); in.h1 = _guess.get(); in.cw = _cw.get();
	in.F0x = _F0x.get(); in.F0y = _F0y.get(); in.F1x = _F1x.get(); in.F1y = _F1y.get(); in.evp = _evpStep.get();
	in.src = _p.on_source ? _src.get() : nullptr;
	in.srcSupplied = _p.src_supplied;
	in.srcConc = _p.src_conc;
}

void Step::ConcAssemble(double dt)
{
	const int nIn = (_p.nx - 4) * (_p.ny - 4);
	ConcIn in;
	ConcInputs(in);
	YZ_LAUNCH(KConcAssemble, GridFor(nIn, 128, 148 * 32), 128, 0, _st, _kc, dt, in, _dRowptrC.get(), _iaC.get(),
	          _rhsC.get());
	if(_bcC.simple)
		YZ_LAUNCH(KConcGhostRhs, GridFor((long long)_ghost.size(), 256), 256, 0, _st, (int)_ghost.size(), _dGhost.get(),
		          _dPartner.get(), _c0.get(), _rhsC.get());
	else
		YZ_LAUNCH(KBcRhs, GridFor((long long)_ghost.size(), 256), 256, 0, _st, (int)_ghost.size(), _dGhost.get(),
		          _dRowptrC.get(), _dColC.get(), _iaC.get(), _dBcCRhs.get(), _c0.get(), _rhsC.get());
}

//  after a converged concentration solve: the ghosts of d by the boundary
//  rows with the d system's right-hand side, c1 = c0 + d, on a committed
//  solve with the advection c1 formed once more from the face fluxes
//  (Reconstruct), c1's ghosts by the rows with the equation's, then the
//  pass's bookkeeping (KConcUpdate)
void Step::ConcUpdate(int mode, double dt)
{
	const int n = _n, g = GridFor(n, 256);
	if(mode == 1 && _kc.conv)
	{
		if(_bcC.simple)
			YZ_LAUNCH(KGhostD, GridFor((long long)_ghost.size(), 256), 256, 0, _st, (int)_ghost.size(), _dGhost.get(),
			          _dPartner.get(), _rhsC.get(), _dC.get());
		else SatisfyConcGhosts(_dC.get(), _rhsC.get());
		YZ_LAUNCH(KAddTo, g, 256, 0, _st, n, _c0.get(), _dC.get(), _cx.get());
		YZ_CUDA(cudaMemcpyAsync(_cPre.get(), _cx.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
		ConcIn in;
		ConcInputs(in);
		const int nIn = (_p.nx - 4) * (_p.ny - 4);
		YZ_LAUNCH(KSoluteFaces, GridFor(nIn, 128), 128, 0, _st, _kc, in, _cPre.get(), _G2x.get(), _G2y.get());
		YZ_LAUNCH(KReconstruct, GridFor(nIn, 256), 256, 0, _st, _kc, dt, in, _cPre.get(), _G2x.get(), _G2y.get(),
		          _cx.get());
		SatisfyConcGhosts(_cx.get(), nullptr);
		YZ_LAUNCH(KConcUpdate, g, 256, 0, _st, n, mode, 1, _dPartnerAll.get(), _c0.get(), _dC.get(), _rhsC.get(),
		          _cx.get(), _cLim.get(), _cw.get(), _cPrev.get(), _red.get() + kSlotCorr);
		return;
	}
	if(_bcC.simple)
	{
		YZ_LAUNCH(KConcUpdate, g, 256, 0, _st, n, mode, 0, _dPartnerAll.get(), _c0.get(), _dC.get(), _rhsC.get(),
		          _cx.get(), _cLim.get(), _cw.get(), _cPrev.get(), _red.get() + kSlotCorr);
		return;
	}
	SatisfyConcGhosts(_dC.get(), _rhsC.get());
	YZ_LAUNCH(KAddTo, g, 256, 0, _st, n, _c0.get(), _dC.get(), _cx.get());
	SatisfyConcGhosts(_cx.get(), nullptr);
	YZ_LAUNCH(KConcUpdate, g, 256, 0, _st, n, mode, 1, _dPartnerAll.get(), _c0.get(), _dC.get(), _rhsC.get(), _cx.get(),
	          _cLim.get(), _cw.get(), _cPrev.get(), _red.get() + kSlotCorr);
}

//  _bcg.Solve of the concentration (ConcEquationBase.h:371): d in/out
int Step::ConcSolve(yz_step_stats &stats)
{
	int it = 0; double res = 0;
	const int r0 = _solverC->Rebuilds();
	int ch;
	{
		YZ_PROF("c.linsolve", _st);
		ch = _solverC->Solve(_p.lin_conc, _iaC.get(), _rhsC.get(), _dC.get(), it, res);
	}
	double su = 0, sit = 0; _solverC->Timing(&su, &sit);
	stats.setup_ms += su; stats.solve_ms += sit;
	stats.amg_setups += _solverC->Rebuilds() - r0;
	stats.conc_iterations += it;
	stats.conc_solves += 1;
	return ch;
}

//  The concentration part of EveryNKLoop (HeightEquationBase.h:1391-1444)
bool Step::ConcPass(double dt, yz_step_stats &stats)
{
	const int n = _n, g = GridFor(n, 256);
	//  the fluxes and the sources of this pass's film, and whether it has a
	//  cell without liquid (then the concentration is left as it is)
	if(FaceFluxes(_guess.get(), _cw.get(), _F1x.get(), _F1y.get(), dt, true)) { _coupled = 0; return true; }
	ConcAssemble(dt);
	const int ch = ConcSolve(stats);
	if(ch != 0) return false;
	ZeroMax(kSlotCorr);
	ConcUpdate(0, dt);
	_coupled = ReadMax(kSlotCorr);
	return true;
}

//  The concentration part of AfterNKLoop (HeightEquationBase.h:1447-1576)
void Step::ConcCommit(double dt, yz_step_stats &stats)
{
	const int n = _n, g = GridFor(n, 256);
	const size_t bytes = (size_t)n * sizeof(double);
	const int nx = _p.nx, ny = _p.ny;
	//  the fluxes at the film the iteration ended on, with the last pass's c;
	//  the evaporation as the last pass's B took it
	const bool noFilm = FaceFluxes(_guess.get(), _cw.get(), _F1x.get(), _F1y.get(), dt, false) != 0;
	YZ_CUDA(cudaMemcpyAsync(_evpStep.get(), _evapB.get(), bytes, cudaMemcpyDeviceToDevice, _st));
	//  ConsistentFluxes: the fluxes of the step the film took
	{
		const int nIn = (nx - 4) * (ny - 4);
		const double w = 1.0 / _p.theta;
		YZ_LAUNCH(KRho, RedBlocks(nIn), kRT, 0, _st, nx, ny, _p.theta, dt, _hOld.get(), _guess.get(), _F1x.get(),
		          _F1y.get(), _F0x.get(), _F0y.get(), _evpStep.get(), _p.on_source ? _src.get() : nullptr, _rho.get(),
		          StepRed(0), _sums.get());
		YZ_LAUNCH(KRowPass, GridFor(ny - 4, 64), 64, 0, _st, nx, ny, w, _rho.get(), _sums.get(), _rowSum.get(),
		          _F1x.get());
		YZ_LAUNCH(KAccY, 1, 32, 0, _st, nx, ny, _rowSum.get(), _accY.get());
		YZ_LAUNCH(KFyFix, GridFor((long long)(nx - 4) * (ny - 5), 256), 256, 0, _st, nx, ny, w, _accY.get(), _F1y.get());
	}
	//  the solve repeated with a limited scheme's limiter frozen at its own
	//  answer until that settles
	YZ_CUDA(cudaMemcpyAsync(_cxLast.get(), _cx.get(), bytes, cudaMemcpyDeviceToDevice, _st));
	const bool limited = _kc.conv && _kc.cI.limited;
	bool solved = true;
	for(int k = 0; k < (limited ? 8 : 1) && !noFilm; ++k)
	{
		ConcAssemble(dt);
		if(ConcSolve(stats) != 0) { solved = false; break; }
		ZeroMax(kSlotCorr);
		ConcUpdate(1, dt);
		if(!limited) break;
		if(ReadMax(kSlotCorr) <= 1e-12) break;
	}
	if(!solved) YZ_CUDA(cudaMemcpyAsync(_cx.get(), _cxLast.get(), bytes, cudaMemcpyDeviceToDevice, _st));
	//  0 <= c <= 1 without taking solute away or making any
	Redistribute();
	//  CommitStep; the working field and the field take c1 capped at 1
	YZ_LAUNCH(KConcCommit, g, 256, 0, _st, n, _cx.get(), _c0.get(), _cw.get(), _cLim.get(), _c.get());
}

//  RedistributeExcess (HeightEquationBase.h:1130-1170) on c1, with the film
//  the step ended on
void Step::Redistribute()
{
	const int n = _n, g = GridFor(n, 256);
	int *flags = _iflags.get() + 1;
	YZ_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), _st));
	YZ_LAUNCH(KExcessFlags, g, 256, 0, _st, n, _dIsbc.get(), _cx.get(), flags);
	int f = 0;
	YZ_CUDA(cudaMemcpyAsync(&f, flags, sizeof(int), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	const bool over = (f & 1) != 0, under = (f & 2) != 0;
	if(over) MoveExcess(false);
	if(under) MoveExcess(true);
	if(over || under) SatisfyConcGhosts(_cx.get(), nullptr);
	YZ_LAUNCH(KBoundRows, g, 256, 0, _st, n, under ? 1 : 0, _cx.get());
}

void Step::MoveExcess(bool lower)
{
	const int n = _n, g = GridFor(n, 256), nx = _p.nx;
	const int lw = lower ? 1 : 0;
	int *flags = _iflags.get() + 2;
	bool any = true;
	for(int pass = 0; pass < 4 && any; ++pass)
	{
		YZ_LAUNCH(KRoom, g, 256, 0, _st, n, lw, _dIsbc.get(), _guess.get(), _cx.get(), _room.get());
		YZ_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), _st));
		YZ_LAUNCH(KOutside, g, 256, 0, _st, nx, n, lw, pass, _dIsbc.get(), _guess.get(), _cx.get(), _room.get(),
		          _give.get(), flags);
		YZ_LAUNCH(KGain, g, 256, 0, _st, nx, n, lw, _dIsbc.get(), _guess.get(), _cx.get(), _room.get(), _give.get(),
		          flags);
		int h = 0;
		YZ_CUDA(cudaMemcpyAsync(&h, flags, sizeof(int), cudaMemcpyDeviceToHost, _st));
		YZ_CUDA(cudaStreamSynchronize(_st));
		any = (h != 0);
	}
	if(!any) return;
	//  what is left: spread over every real cell with room, in proportion
	YZ_LAUNCH(KSpreadSums, RedBlocks(n), kRT, 0, _st, n, lw, _dIsbc.get(), _guess.get(), _cx.get(), StepRed(1),
	          _sums.get() + 2);
	double sums[2] = {0, 0};
	YZ_CUDA(cudaMemcpyAsync(sums, _sums.get() + 2, sizeof sums, cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	const double left = sums[0], total = sums[1];
	const double f = (total > 0.0) ? std::min(1.0, left / total) : 0.0;
	if(f > 0.0) YZ_LAUNCH(KSpreadApply, g, 256, 0, _st, n, lw, _dIsbc.get(), _guess.get(), _cx.get(), f);
}

int Step::ConcPattern(int *rowptr, int *col) const
{
	if(!_conc) return 0;
	if(rowptr) std::copy(_rowptrC.begin(), _rowptrC.end(), rowptr);
	if(col) std::copy(_colC.begin(), _colC.end(), col);
	return _nnzC;
}

//  The first pass's concentration system of a step from (h, c): h1 = h0 = h,
//  F1 = F0, the limiter and the working field's c at c
void Step::ConcSystem(const double *h, const double *c, double dt, double *val, double *rhs)
{
	if(!_conc) throw UsageError("step: the case has no concentration equation (conc_field = 0)");
	YZ_CUDA(cudaSetDevice(_device));
	const size_t bytes = (size_t)_n * sizeof(double);
	YZ_CUDA(cudaMemcpyAsync(_hOld.get(), h, bytes, cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_guess.get(), h, bytes, cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_c0.get(), c, bytes, cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_cw.get(), c, bytes, cudaMemcpyHostToDevice, _st));
	YZ_CUDA(cudaMemcpyAsync(_cLim.get(), c, bytes, cudaMemcpyHostToDevice, _st));
	if(_p.on_source) UpdateSource(dt);
	//  evapOld at h (mode 0 of the assembly), then the pass's fluxes and sources
	Assemble(0, _hOld.get(), _cw.get(), dt);
	FaceFluxes(_hOld.get(), _cw.get(), _F0x.get(), _F0y.get(), dt, false);
	FaceFluxes(_guess.get(), _cw.get(), _F1x.get(), _F1y.get(), dt, true);
	ConcAssemble(dt);
	_iaC.download(val, (size_t)_nnzC, _st);
	_rhsC.download(rhs, (size_t)_n, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

} // namespace yz
