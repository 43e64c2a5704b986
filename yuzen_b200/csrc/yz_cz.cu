// yz_cz.cu -- the ConcZ model's time step on the device (see yz_cz.h).
#include "yz_cz.h"
#include "yz_exp.h"
#include "yz_prof.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace yz {

using namespace phys;

namespace {

constexpr int kB = 256;
enum { kBcSym = 0, kBcPer = 1, kBcPin = 2 };

__host__ __device__ __forceinline__ int I2(const CzCoef &k, int ix, int jy) { return jy * k.nx + ix; }
__host__ __device__ __forceinline__ int I3(const CzCoef &k, int ix, int jy, int kz) { return (kz * k.ny + jy) * k.nx + ix; }

//  the property laws (FluidProperty.h:176-180) with the correctly rounded exp
//  (yz_exp.h), the one the ConcZ oracle links too
__device__ __forceinline__ double Diff(const CzCoef &k, double c)
{
	return k.diffBase * crexp::Exp(k.diffExp * (c - k.diffC0));
}
__device__ __forceinline__ double ViscCz(const CzCoef &k, double c)
{
	return k.ev.viscBase * crexp::Exp(k.ev.viscExp * (c - k.ev.viscC0));
}

//  |v| into a running maximum (non-negative doubles order as their bits);
//  every lane of the warp takes part
__device__ __forceinline__ void MaxAbsInto(unsigned long long *slot, double v)
{
	unsigned long long u = (unsigned long long)__double_as_longlong(fabs(v));
	for(int off = 16; off >= 1; off >>= 1)
	{
		const unsigned long long w = __shfl_down_sync(0xffffffffu, u, off);
		u = w > u ? w : u;
	}
	if((threadIdx.x & 31) == 0 && u) atomicMax(slot, u);
}

//==========================================================================
//  The film's faces
//==========================================================================
//  FaceInvViscosity (CZ_HeightEquation_2D.cpp:624-640): the mean of 1/mu
//  through the film at the face below (ix, jy) along (ax, ay), weighted by
//  (1 - zeta)^power, over the real levels
__device__ double FaceInvVisc(const CzCoef &k, const double *C, int ix, int jy, int ax, int ay, int power)
{
	double num = 0, den = 0;
	for(int kz = 2; kz < k.nz - 2; ++kz)
	{
		const double c = 0.5 * (C[I3(k, ix - ax, jy - ay, kz)] + C[I3(k, ix, jy, kz)]);
		const double r = 1.0 - k.dzeta * (-1.5 + (double)kz);
		const double w = (power == 2) ? r * r : r;
		num += w / ViscCz(k, c);
		den += w;
	}
	return num / den;
}

//  WallFace (:672-679)
__device__ __forceinline__ bool WallFaceCz(const CzCoef &k, int ix, int jy, int ax)
{
	if(ax) return (ix == 2 && k.wall[0]) || (ix == k.nx - 2 && k.wall[1]);
	return (jy == 2 && k.wall[2]) || (jy == k.ny - 2 && k.wall[3]);
}

//  per face of either axis (x faces ix = 2 .. nx-2 of the real rows, y faces
//  jy = 2 .. ny-2 of the real columns, held at IL(ix, jy)): FaceMobility
//  (:681-714), the surface tension of FaceSurfConc (:648-655), MarangoniFlux
//  (:716-748), and the capillary coefficient and explicit rest of the face
//  flux (StoreFaceFluxParts, :1161-1230)
__global__ void KCzFaces(CzCoef k, const double *__restrict__ H, const double *__restrict__ S,
                         const double *__restrict__ C, double *Dx, double *Sgx, double *Mx, double *capx, double *expx,
                         double *Dy, double *Sgy, double *My, double *capy, double *expy)
{
	const int fx = (k.nx - 3) * (k.ny - 4), fy = (k.nx - 4) * (k.ny - 3);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < fx + fy; t += gridDim.x * blockDim.x)
	{
		const bool xa = t < fx;
		int ix, jy;
		if(xa) { ix = 2 + t % (k.nx - 3); jy = 2 + t / (k.nx - 3); }
		else { const int u = t - fx; ix = 2 + u % (k.nx - 4); jy = 2 + u / (k.nx - 4); }
		const int ax = xa ? 1 : 0, ay = xa ? 0 : 1;
		auto Hh = [&](int i, int j) { return H[I2(k, i, j)]; };
		auto Ss = [&](int i, int j) { return S[I2(k, i, j)]; };
		const double h1 = Hh(ix - ax, jy - ay), h2 = Hh(ix, jy);
		const bool wall = WallFaceCz(k, ix, jy, ax);
		//  FaceMobility
		double D = 0.0;
		if(!wall)
		{
			const double denom = h1 + h2;
			if(denom > 0.0)
			{
				const double mob = 2.0 * (h1 * h1) * (h2 * h2) / denom;
				D = mob / 3.0 * FaceInvVisc(k, C, ix, jy, ax, ay, 2);
			}
		}
		//  the surface tension of the face's surface concentration
		const int zt = k.nz - 2, zr = k.nz - 3;
		const double cs = 0.25 * (C[I3(k, ix - ax, jy - ay, zt)] + C[I3(k, ix - ax, jy - ay, zr)] +
		                          C[I3(k, ix, jy, zt)] + C[I3(k, ix, jy, zr)]);
		const double sig = SurfaceTension(k.ev, cs);
		//  MarangoniFlux
		double M = 0.0;
		if(k.onSC && !wall && !(h1 + h2 <= 0.0))
		{
			const double ds = xa ? k.dx : k.dy;
			const double cs1 = 0.5 * (C[I3(k, ix - ax, jy - ay, zt)] + C[I3(k, ix - ax, jy - ay, zr)]);
			const double cs2 = 0.5 * (C[I3(k, ix, jy, zt)] + C[I3(k, ix, jy, zr)]);
			const double dcds = (cs2 - cs1) / ds;
			const double h2eff = h1 * h2;
			M = 0.5 * h2eff * k.As * k.Ma * dcds * FaceInvVisc(k, C, ix, jy, ax, ay, 1);
		}
		//  StoreFaceFluxParts
		double cap = 0.0, expl = 0.0;
		if(xa)
		{
			if(k.onL)
			{
				cap = D * sig;
				double d3s = (Ss(ix + 1, jy) - 3.0 * Ss(ix, jy) + 3.0 * Ss(ix - 1, jy) - Ss(ix - 2, jy)) * k.rdx * k.rdx2;
				d3s += ((Ss(ix, jy + 1) - 2.0 * Ss(ix, jy) + Ss(ix, jy - 1)) -
				        (Ss(ix - 1, jy + 1) - 2.0 * Ss(ix - 1, jy) + Ss(ix - 1, jy - 1))) * k.rdx * k.rdy2;
				expl += cap * d3s;
			}
			if(k.onVG) expl -= D * k.Bo * ((Hh(ix, jy) + Ss(ix, jy)) - (Hh(ix - 1, jy) + Ss(ix - 1, jy))) * k.rdx;
			if(k.onHG) expl += D * k.Pgx;
			if(k.onCF) expl += D * k.Sp * (k.xf[ix] - k.rot0);
			if(k.onSC) expl += M;
			const int o = I2(k, ix, jy);
			Dx[o] = D; Sgx[o] = sig; Mx[o] = M; capx[o] = cap; expx[o] = expl;
		}
		else
		{
			if(k.onL)
			{
				cap = D * sig;
				double d3s = (Ss(ix, jy + 1) - 3.0 * Ss(ix, jy) + 3.0 * Ss(ix, jy - 1) - Ss(ix, jy - 2)) * k.rdy * k.rdy2;
				d3s += ((Ss(ix - 1, jy) - 2.0 * Ss(ix, jy) + Ss(ix + 1, jy)) -
				        (Ss(ix - 1, jy - 1) - 2.0 * Ss(ix, jy - 1) + Ss(ix + 1, jy - 1))) * k.rdy * k.rdx2;
				expl += cap * d3s;
			}
			if(k.onVG) expl -= D * k.Bo * ((Hh(ix, jy) + Ss(ix, jy)) - (Hh(ix, jy - 1) + Ss(ix, jy - 1))) * k.rdy;
			if(k.onHG) expl += D * k.Pgy;
			if(k.onCF) expl += D * k.Sp * (k.yf[jy] - k.rot1);
			if(k.onSC) expl += M;
			const int o = I2(k, ix, jy);
			Dy[o] = D; Sgy[o] = sig; My[o] = M; capy[o] = cap; expy[o] = expl;
		}
	}
}

//  ColumnMeanConc (:388-393)
__device__ __forceinline__ double ColumnMean(const CzCoef &k, const double *C, int ix, int jy)
{
	double s = 0.0;
	for(int kz = 2; kz < k.nz - 2; ++kz) s += C[I3(k, ix, jy, kz)];
	return s / (double)(k.nz - 4);
}

//  C_Evaporation::SolventLimit (Evaporation.h:112-119)
__device__ __forceinline__ double SolventLimitCz(double evp, double h, double c, double dt)
{
	if(!(evp > 0.0)) return evp;
	const double cc = (c < 0.0) ? 0.0 : ((c > 1.0) ? 1.0 : c);
	const double solvent = (h > 0.0) ? h * (1.0 - cc) : 0.0;
	if(evp * dt > solvent) evp = solvent / dt;
	return evp;
}

//  the evaporation rate of a column at the surface concentration of C
//  (C_Evaporation::operator()(Field_CZ&, Zface), Evaporation.cpp:143-169)
__device__ __forceinline__ double EvapCol(const CzCoef &k, const double *H, const double *C, int ix, int jy)
{
	const double cc = 0.5 * (C[I3(k, ix, jy, k.nz - 3)] + C[I3(k, ix, jy, k.nz - 2)]);
	return k.Ev * EvapRate(k.ev, H[I2(k, ix, jy)], cc, k.xc[ix], k.yc[jy]);
}

//==========================================================================
//  The film's rows (SetMatrixA, CZ_HeightEquation_2D.cpp:750-1050): one
//  thread per real row; its 13 values in storage order (the diagonal, x-2,
//  x-1, x+1, x+2, y-2, y-1, y+1, y+2, (-1,-1), (-1,+1), (+1,-1), (+1,+1)),
//  the right-hand side B = -h_t and the column's source
//==========================================================================
__global__ void KCzAssembleH(CzCoef k, const int *__restrict__ rowptr, const double *__restrict__ H,
                             const double *__restrict__ S, const double *__restrict__ C, const double *__restrict__ HT,
                             const double *__restrict__ CT, const double *__restrict__ Dx, const double *__restrict__ Sgx,
                             const double *__restrict__ Mx, const double *__restrict__ Dy, const double *__restrict__ Sgy,
                             const double *__restrict__ My, double dt, double *A, double *B, double *colSrc)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + t / rx;
		const int row = I2(k, ix, jy);
		auto Hh = [&](int i, int j) { return H[I2(k, i, j)]; };
		auto Ss = [&](int i, int j) { return S[I2(k, i, j)]; };
		const double DL = Dx[I2(k, ix, jy)], DR = Dx[I2(k, ix + 1, jy)];
		const double sigL = Sgx[I2(k, ix, jy)], sigR = Sgx[I2(k, ix + 1, jy)];
		const double aL = k.onL ? DL * sigL * k.rdx4 : 0.0;
		const double aR = k.onL ? DR * sigR * k.rdx4 : 0.0;
		const double DB = Dy[I2(k, ix, jy)], DT = Dy[I2(k, ix, jy + 1)];
		const double sigB = Sgy[I2(k, ix, jy)], sigT = Sgy[I2(k, ix, jy + 1)];
		const double bB = k.onL ? DB * sigB * k.rdy4 : 0.0;
		const double bT = k.onL ? DT * sigT * k.rdy4 : 0.0;
		const double cL = k.onL ? DL * sigL * k.rdx2dy2 : 0.0;
		const double cR = k.onL ? DR * sigR * k.rdx2dy2 : 0.0;
		const double cB = k.onL ? DB * sigB * k.rdx2dy2 : 0.0;
		const double cT = k.onL ? DT * sigT * k.rdx2dy2 : 0.0;
		double *a = A + rowptr[row];
		double dg = +3.0 * aL + 3.0 * aR;
		dg += +3.0 * bB + 3.0 * bT;
		dg += +2.0 * cL + 2.0 * cR;
		dg += +2.0 * cB + 2.0 * cT;
		a[0] = dg;
		a[1] = +aL;
		double v = -3.0 * aL - aR;
		v += -2.0 * cL;
		v += -cB - cT;
		a[2] = v;
		v = -aL - 3.0 * aR;
		v += -2.0 * cR;
		v += -cB - cT;
		a[3] = v;
		a[4] = +aR;
		a[5] = 0.0 + bB;
		v = 0.0;
		v += -3.0 * bB - bT;
		v += -cL - cR;
		v += -2.0 * cB;
		a[6] = v;
		v = 0.0;
		v += -bB - 3.0 * bT;
		v += -cL - cR;
		v += -2.0 * cT;
		a[7] = v;
		a[8] = 0.0 + bT;
		v = 0.0; v += +cL; v += +cB; a[9] = v;
		v = 0.0; v += +cL; v += +cT; a[10] = v;
		v = 0.0; v += +cR; v += +cB; a[11] = v;
		v = 0.0; v += +cR; v += +cT; a[12] = v;

		//  the right-hand side, as h_t first
		const double sPo = Ss(ix + 2, jy), spo = Ss(ix + 1, jy), smo = Ss(ix - 1, jy), sMo = Ss(ix - 2, jy);
		const double soo = Ss(ix, jy);
		const double rdx = k.rdx, rdx2 = k.rdx2, rdy = k.rdy, rdy2 = k.rdy2;
		double dhdt = 0.0;
		if(k.onL)
		{
			const double d3sL = (spo - 3.0 * soo + 3.0 * smo - sMo) * rdx * rdx2;
			const double d3sR = (sPo - 3.0 * spo + 3.0 * soo - smo) * rdx * rdx2;
			dhdt -= (DR * sigR * d3sR - DL * sigL * d3sL) * rdx;
		}
		if(k.onVG)
		{
			const double hsP = Hh(ix + 1, jy) + spo;
			const double hsO = Hh(ix, jy) + soo;
			const double hsM = Hh(ix - 1, jy) + smo;
			const double gR = DR * k.Bo * (hsP - hsO) * rdx;
			const double gL = DL * k.Bo * (hsO - hsM) * rdx;
			dhdt += (gR - gL) * rdx;
		}
		if(k.onHG)
		{
			const double fR = DR * k.Pgx;
			const double fL = DL * k.Pgx;
			dhdt -= (fR - fL) * rdx;
		}
		if(k.onCF)
		{
			const double xR = k.xf[ix + 1] - k.rot0;
			const double xL = k.xf[ix] - k.rot0;
			dhdt -= (DR * k.Sp * xR - DL * k.Sp * xL) * rdx;
		}
		if(k.onSC) dhdt -= (Mx[I2(k, ix + 1, jy)] - Mx[I2(k, ix, jy)]) * rdx;
		{
			if(k.onL)
			{
				const double soP = Ss(ix, jy + 2), sop = Ss(ix, jy + 1), som = Ss(ix, jy - 1), soM = Ss(ix, jy - 2);
				const double d3sB = (sop - 3.0 * soo + 3.0 * som - soM) * rdy * rdy2;
				const double d3sT = (soP - 3.0 * sop + 3.0 * soo - som) * rdy * rdy2;
				dhdt -= (DT * sigT * d3sT - DB * sigB * d3sB) * rdy;
				const double smm = Ss(ix - 1, jy - 1), smp = Ss(ix - 1, jy + 1);
				const double spm = Ss(ix + 1, jy - 1), spp = Ss(ix + 1, jy + 1);
				const double xL_ = ((som - 2.0 * soo + sop) - (smm - 2.0 * smo + smp)) * rdx * rdy2;
				const double xR_ = ((spm - 2.0 * spo + spp) - (som - 2.0 * soo + sop)) * rdx * rdy2;
				dhdt -= (DR * sigR * xR_ - DL * sigL * xL_) * rdx;
				const double yB_ = ((smo - 2.0 * soo + spo) - (smm - 2.0 * som + spm)) * rdy * rdx2;
				const double yT_ = ((smp - 2.0 * sop + spp) - (smo - 2.0 * soo + spo)) * rdy * rdx2;
				dhdt -= (DT * sigT * yT_ - DB * sigB * yB_) * rdy;
			}
			if(k.onVG)
			{
				const double sop = Ss(ix, jy + 1), som = Ss(ix, jy - 1);
				const double hsT = Hh(ix, jy + 1) + sop;
				const double hsO = Hh(ix, jy) + soo;
				const double hsB = Hh(ix, jy - 1) + som;
				const double gT = DT * k.Bo * (hsT - hsO) * rdy;
				const double gB = DB * k.Bo * (hsO - hsB) * rdy;
				dhdt += (gT - gB) * rdy;
			}
			if(k.onHG) dhdt -= (DT * k.Pgy - DB * k.Pgy) * rdy;
			if(k.onCF)
			{
				const double yT = k.yf[jy + 1] - k.rot1;
				const double yB = k.yf[jy] - k.rot1;
				dhdt -= (DT * k.Sp * yT - DB * k.Sp * yB) * rdy;
			}
			if(k.onSC) dhdt -= (My[I2(k, ix, jy + 1)] - My[I2(k, ix, jy)]) * rdy;
		}
		//  evaporation, no more than the solvent the column holds now and at
		//  the start of the step
		double Evap = k.onEvap ? EvapCol(k, H, C, ix, jy) : 0.0;
		if(Evap > 0.0)
		{
			Evap = SolventLimitCz(Evap, Hh(ix, jy), ColumnMean(k, C, ix, jy), dt);
			Evap = SolventLimitCz(Evap, HT[row], ColumnMean(k, CT, ix, jy), dt);
		}
		dhdt -= Evap;
		colSrc[row] = 0.0 - Evap - 0.0;
		B[row] = -dhdt;
	}
}

//  MakeMatrix_IA (SemiImplicit.cpp:161-183) on the real rows; the ghost rows
//  of IA are the copies of A's, written once
__global__ void KCzMakeIA(int n, const int *__restrict__ rowptr, const unsigned char *__restrict__ bc,
                          const double *__restrict__ A, double *IA, double theta, double dt)
{
	for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
	{
		if(bc[r]) continue;
		const int st = rowptr[r], ed = rowptr[r + 1];
		IA[st] = 1.0 + theta * dt * A[st];
		for(int q = st + 1; q < ed; ++q) IA[q] = theta * dt * A[q];
	}
}

//  CRS_Matrix::MatVec (CRS_Matrix.cpp:307-329): each row in storage order
__global__ void KCzMatVec(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                          const double *__restrict__ A, const double *__restrict__ x, double *y)
{
	for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
	{
		double sum = 0.0;
		const int ed = rowptr[r + 1];
		for(int q = rowptr[r]; q < ed; ++q) sum += A[q] * x[col[q]];
		y[r] = sum;
	}
}

//  MakeRHS (SemiImplicit.cpp:185-196); the ghost rows' right-hand side stays 0
__global__ void KCzMakeRhsH(int n, const unsigned char *__restrict__ bc, const double *__restrict__ old,
                            const double *__restrict__ Ax, const double *__restrict__ B, double theta, double dt,
                            double *rhs)
{
	for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
		if(!bc[r]) rhs[r] = old[r] - dt * (1.0 - theta) * Ax[r] - dt * B[r];
}

} // namespace

namespace {

//==========================================================================
//  The film's ghosts and its conservative update
//==========================================================================
//  CopyGhosts (:1346-1360): the ghost rows are copies ([1, -1], right-hand
//  side 0); the y ghosts of the real columns first, then the x ghosts of
//  every row (a corner reads a y ghost), which is where the reference's two
//  sweeps in row order end up
__global__ void KCzGhostY(CzCoef k, double *h)
{
	const int rx = k.nx - 4;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < rx * 4; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, g = t / rx;
		const int jy = g < 2 ? g : k.ny - 4 + g;            // 0, 1, ny-2, ny-1
		int p;
		if(k.perY) p = (jy == 0) ? k.ny - 4 : (jy == 1) ? k.ny - 3 : (jy == k.ny - 2) ? 2 : 3;
		else p = (jy == 0) ? 3 : (jy == 1) ? 2 : (jy == k.ny - 2) ? k.ny - 3 : k.ny - 4;
		h[I2(k, ix, jy)] = h[I2(k, ix, p)];
	}
}
__global__ void KCzGhostX(CzCoef k, double *h)
{
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < k.ny * 4; t += gridDim.x * blockDim.x)
	{
		const int jy = t % k.ny, g = t / k.ny;
		const int ix = g < 2 ? g : k.nx - 4 + g;
		int p;
		if(k.perX) p = (ix == 0) ? k.nx - 4 : (ix == 1) ? k.nx - 3 : (ix == k.nx - 2) ? 2 : 3;
		else p = (ix == 0) ? 3 : (ix == 1) ? 2 : (ix == k.nx - 2) ? k.nx - 3 : k.nx - 4;
		h[I2(k, ix, jy)] = h[I2(k, p, jy)];
	}
}

//  ConservativeUpdate (:1232-1301): the flux of every face with the
//  Crank-Nicolson h of the solve (hc = theta h_new + (1 - theta) h_old)
__global__ void KCzFaceFlux(CzCoef k, const double *__restrict__ hc, const double *__restrict__ capx,
                            const double *__restrict__ expx, const double *__restrict__ capy,
                            const double *__restrict__ expy, double *qx, double *qy)
{
	const int fx = (k.nx - 3) * (k.ny - 4), fy = (k.nx - 4) * (k.ny - 3);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < fx + fy; t += gridDim.x * blockDim.x)
	{
		auto Hc = [&](int i, int j) { return hc[I2(k, i, j)]; };
		if(t < fx)
		{
			const int ix = 2 + t % (k.nx - 3), jy = 2 + t / (k.nx - 3);
			double d3h = (Hc(ix + 1, jy) - 3.0 * Hc(ix, jy) + 3.0 * Hc(ix - 1, jy) - Hc(ix - 2, jy)) * k.rdx * k.rdx2;
			d3h += ((Hc(ix, jy + 1) - 2.0 * Hc(ix, jy) + Hc(ix, jy - 1)) -
			        (Hc(ix - 1, jy + 1) - 2.0 * Hc(ix - 1, jy) + Hc(ix - 1, jy - 1))) * k.rdx * k.rdy2;
			const int o = I2(k, ix, jy);
			qx[o] = capx[o] * d3h + expx[o];
		}
		else
		{
			const int u = t - fx, ix = 2 + u % (k.nx - 4), jy = 2 + u / (k.nx - 4);
			double d3h = (Hc(ix, jy + 1) - 3.0 * Hc(ix, jy) + 3.0 * Hc(ix, jy - 1) - Hc(ix, jy - 2)) * k.rdy * k.rdy2;
			d3h += ((Hc(ix - 1, jy) - 2.0 * Hc(ix, jy) + Hc(ix + 1, jy)) -
			        (Hc(ix - 1, jy - 1) - 2.0 * Hc(ix, jy - 1) + Hc(ix + 1, jy - 1))) * k.rdy * k.rdx2;
			const int o = I2(k, ix, jy);
			qy[o] = capy[o] * d3h + expy[o];
		}
	}
}

__global__ void KCzHc(int n, const double *__restrict__ hNew, const double *__restrict__ hOld, double theta, double *hc)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double a = hNew[i] * theta;
		const double b = hOld[i] * (1.0 - theta);
		hc[i] = a + b;
	}
}

__global__ void KCzEnd(CzCoef k, const double *__restrict__ hOld, const double *__restrict__ qx,
                       const double *__restrict__ qy, const double *__restrict__ colSrc, double dt, double *hNew)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + t / rx, o = I2(k, ix, jy);
		double div = (qx[I2(k, ix + 1, jy)] - qx[o]) * k.rdx;
		div += (qy[I2(k, ix, jy + 1)] - qy[o]) * k.rdy;
		hNew[o] = hOld[o] + dt * (colSrc[o] - div);
	}
}

//  CalDtDh (:1362-1367)
__global__ void KCzDtDh(int n, const double *__restrict__ hNew, const double *__restrict__ hOld, double dt, double *dtdh)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		double v = hNew[i];
		v -= hOld[i];
		dtdh[i] = v / dt;
	}
}

//==========================================================================
//  CalVelocity (:1381-1790): the in-plane velocity through the film,
//  Simpson's rule of 1/mu and z/mu from the substrate up, times the driving
//  force of each term; one thread per face column
//==========================================================================
template<int AX>
__global__ void KCzVel(CzCoef k, const double *__restrict__ H, const double *__restrict__ S,
                       const double *__restrict__ C, double *U)
{
	//  x faces: ix = 2 .. nx-2 of every row; y faces: jy = 2 .. ny-2 of every column
	const int na = AX ? (k.nx - 3) : k.nx, nb = AX ? k.ny : (k.ny - 3);
	const int sz = k.nx * k.ny;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < na * nb; t += gridDim.x * blockDim.x)
	{
		const int ix = AX ? 2 + t % na : t % na;
		const int jy = AX ? t / na : 2 + t / na;
		const int ax = AX ? 1 : 0, ay = AX ? 0 : 1;
		auto Hh = [&](int i, int j) { return H[I2(k, i, j)]; };
		auto Ss = [&](int i, int j) { return S[I2(k, i, j)]; };
		auto Cc = [&](int i, int j, int q) { return C[I3(k, i, j, q)]; };
		const double hpo = Hh(ix + ax, jy + ay), hoo = Hh(ix, jy), hmo = Hh(ix - ax, jy - ay), hMo = Hh(ix - 2 * ax, jy - 2 * ay);
		const double spo = Ss(ix + ax, jy + ay), soo = Ss(ix, jy), smo = Ss(ix - ax, jy - ay), sMo = Ss(ix - 2 * ax, jy - 2 * ay);
		const double hL = 0.5 * (hmo + hoo);
		const double sL = 0.5 * (smo + soo);
		const double xL = AX ? k.xf[ix] - k.rot0 : k.yf[jy] - k.rot1;
		const int zt = k.nz - 2, zr = k.nz - 3;
		const double Cpoo = Cc(ix + ax, jy + ay, zt), Cooo0 = Cc(ix, jy, zt), Cmoo0 = Cc(ix - ax, jy - ay, zt),
		             CMoo = Cc(ix - 2 * ax, jy - 2 * ay, zt);
		const double Cpom = Cc(ix + ax, jy + ay, zr), Coom0 = Cc(ix, jy, zr), Cmom0 = Cc(ix - ax, jy - ay, zr),
		             CMom = Cc(ix - 2 * ax, jy - 2 * ay, zr);
		const double dd = AX ? k.dx : k.dy;
		const double dcdx_suf = 0.5 * ((-Cpoo + 27.0 * Cooo0 - 27.0 * Cmoo0 + CMoo) +
		                               (-Cpom + 27.0 * Coom0 - 27.0 * Cmom0 + CMom)) / (24.0 * dd);
		const double dx3hs = ((hpo + spo) - 3.0 * (hoo + soo) + 3.0 * (hmo + smo) - (hMo + sMo)) / (AX ? k.dx3 : k.dy3);
		const double dxhs = (-(hpo + spo) + 27.0 * (hoo + soo) - 27.0 * (hmo + smo) + (hMo + sMo)) / (24.0 * dd);
		const double sigma = SurfaceTension(k.ev, 0.25 * (Cooo0 + Coom0 + Cmoo0 + Cmom0));

		double Cooo = Cc(ix, jy, 2), Cmoo = Cc(ix - ax, jy - ay, 2);
		double Coom = Cc(ix, jy, 1), Cmom = Cc(ix - ax, jy - ay, 1);
		const double muB = ViscCz(k, 0.25 * (Cooo + Coom + Cmoo + Cmom));
		double fB1 = 1.0 / muB;
		double fB2 = sL / muB;
		const double dz = k.dzeta * hL;
		double sum1 = 0, sum2 = 0;
		//  the cross term d^3/(dx dy^2) (d^3/(dy dx^2) at a y face), from the
		//  rows (columns) either side
		double cross = 0.0;
		if(AX ? (jy >= 1 && jy <= k.ny - 2) : (ix >= 1 && ix <= k.nx - 2))
		{
			const double oo2 = AX ? k.dy * k.dy : k.dx * k.dx;
			const int bx = AX ? 0 : 1, by = AX ? 1 : 0;
			const double fOp = Hh(ix + bx, jy + by) + Ss(ix + bx, jy + by);
			const double fOm = Hh(ix - bx, jy - by) + Ss(ix - bx, jy - by);
			const double fMp = Hh(ix - ax + bx, jy - ay + by) + Ss(ix - ax + bx, jy - ay + by);
			const double fMm = Hh(ix - ax - bx, jy - ay - by) + Ss(ix - ax - bx, jy - ay - by);
			cross = ((fOp - 2.0 * (hoo + soo) + fOm) - (fMp - 2.0 * (hmo + smo) + fMm)) / (dd * oo2);
		}
		const double kLap = k.onL ? sigma * (dx3hs + cross) : 0.0;
		const double kMa = k.onSC ? k.As * k.Ma * dcdx_suf : 0.0;
		const double kBo = k.onVG ? -k.Bo * dxhs : 0.0;
		const double kPg = k.onHG ? (AX ? k.Pgx : k.Pgy) : 0.0;
		const double kSp = k.onCF ? k.Sp * xL : 0.0;
		const double hLsL = hL + sL;
		const int o = I2(k, ix, jy);
		for(int kz = 2; kz < k.nz; ++kz)
		{
			const double zT = sL + dz * (-1.5 + (double)kz);
			const double zM = (kz == 2) ? sL + 0.25 * dz : sL + dz * (-2.0 + (double)kz);
			if(kz > 2)
			{
				Coom = Cooo;
				Cmom = Cmoo;
				Cooo = Cc(ix, jy, kz);
				Cmoo = Cc(ix - ax, jy - ay, kz);
			}
			const double muM = (kz == 2) ? ViscCz(k, 0.375 * (Cooo + Cmoo) + 0.125 * (Coom + Cmom))
			                             : ViscCz(k, 0.25 * (Cooo + Coom + Cmoo + Cmom));
			const double muT = ViscCz(k, 0.50 * (Cooo + Cmoo));
			const double fT1 = 1.0 / muT;
			const double fT2 = zT / muT;
			const double fM1 = 1.0 / muM;
			const double fM2 = zM / muM;
			double dz_tmp = dz;
			if(kz == 2) dz_tmp = 0.5 * dz;
			sum1 += (fB1 + fT1 + 4.0 * fM1) * dz_tmp / 6.0;
			sum2 += (fB2 + fT2 + 4.0 * fM2) * dz_tmp / 6.0;
			fB1 = fT1;
			fB2 = fT2;
			const double PP = hLsL * sum1 - sum2;
			double uu = 0;
			if(k.onL) uu += kLap * PP;
			if(k.onSC) uu += kMa * sum1;
			if(k.onVG) uu += kBo * PP;
			if(k.onHG) uu += kPg * PP;
			if(k.onCF) uu += kSp * PP;
			U[o + kz * sz] = uu;
		}
		//  below the substrate: no slip
		U[o] = 0;
		U[o + sz] = -U[o + 2 * sz];
	}
}

//  the velocity outside the walls / across the seams, per row (x) or
//  column (y) and level (:1700-1790)
template<int AX>
__global__ void KCzVelGhost(CzCoef k, double *U)
{
	const int nl = AX ? k.ny : k.nx, n = nl * k.nz;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		const int l = t % nl, kz = t / nl;
		const int N = AX ? k.nx : k.ny;
		auto at = [&](int a) -> double & { return AX ? U[I3(k, a, l, kz)] : U[I3(k, l, a, kz)]; };
		if(AX ? k.perXv : k.perYv)
		{
			at(1) = at(N - 3);
			at(0) = at(N - 4);
			at(N - 1) = at(3);
		}
		else
		{
			if(AX ? WallFaceCz(k, 2, l, 1) : WallFaceCz(k, l, 2, 0)) at(2) = 0.0;
			if(AX ? WallFaceCz(k, N - 2, l, 1) : WallFaceCz(k, l, N - 2, 0)) at(N - 2) = 0.0;
			at(1) = -at(3);
			at(0) = -at(4);
			at(N - 1) = -at(N - 3);
		}
	}
}

//==========================================================================
//  BuildVolumeFluxes (CZ_ConcEquation_2D.cpp:135-272)
//==========================================================================
//  the layer fluxes of one face: the film at the face times the cell mean
//  of the velocity profile, made to add up to the film's face flux
__global__ void KCzLayerFlux(CzCoef k, const double *__restrict__ H, const double *__restrict__ Ux,
                             const double *__restrict__ Uy, const double *__restrict__ qx,
                             const double *__restrict__ qy, double *Qx, double *Qy)
{
	const int fx = (k.nx - 3) * (k.ny - 4), fy = (k.nx - 4) * (k.ny - 3);
	const int sz = k.nx * k.ny;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < fx + fy; t += gridDim.x * blockDim.x)
	{
		const bool xa = t < fx;
		int ix, jy;
		if(xa) { ix = 2 + t % (k.nx - 3); jy = 2 + t / (k.nx - 3); }
		else { const int u = t - fx; ix = 2 + u % (k.nx - 4); jy = 2 + u / (k.nx - 4); }
		const int o = I2(k, ix, jy);
		const double *U = xa ? Ux : Uy;
		double *Q = xa ? Qx : Qy;
		const double hf = xa ? 0.5 * (H[I2(k, ix - 1, jy)] + H[o]) : 0.5 * (H[I2(k, ix, jy - 1)] + H[o]);
		const int k0 = 2, k1 = k.nz - 3;
		double sum = 0.0;
		for(int kz = k0; kz <= k1; ++kz)
		{
			const double u = U[o + kz * sz], up = U[o + (kz + 1) * sz];
			double um;
			if(kz == k0) um = u + (up - 3.0 * u) / 18.0;
			else um = u + (up - 2.0 * u + U[o + (kz - 1) * sz]) / 24.0;
			const double q = hf * um;
			Q[o + kz * sz] = q;
			sum += q * k.dzeta;
		}
		const double d = (xa ? qx[o] : qy[o]) - sum;
		for(int kz = k0; kz <= k1; ++kz) Q[o + kz * sz] += d;
	}
}

//  the zeta faces of every real column, from the substrate up; the free
//  surface takes what leaves the column there (its source)
__global__ void KCzZetaFlux(CzCoef k, const double *__restrict__ dtdh, const double *__restrict__ Qx,
                            const double *__restrict__ Qy, const double *__restrict__ colSrc, double *W)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4), sz = k.nx * k.ny;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + t / rx, o = I2(k, ix, jy);
		const double ht = dtdh[o];
		double w = 0.0;
		W[o + 2 * sz] = 0.0;
		for(int kz = 2; kz < k.nz - 2; ++kz)
		{
			double div = ht + (Qx[o + 1 + kz * sz] - Qx[o + kz * sz]) / k.dx;
			div += (Qy[o + k.nx + kz * sz] - Qy[o + kz * sz]) / k.dy;
			w -= k.dzeta * div;
			W[o + (kz + 1) * sz] = w;
		}
		W[o + (k.nz - 2) * sz] = -(colSrc[o] + 0.0);
	}
}

} // namespace

namespace {

//==========================================================================
//  The concentration's rows (SetMatrixA, CZ_ConcEquation_2D.cpp:301-587):
//  one thread per real cell; its 21 values in storage order (the diagonal,
//  then (0,-2) (-1,-1) (0,-1) (+1,-1) (-2,0) (-1,0) (+1,0) (+2,0) (-1,+1)
//  (0,+1) (+1,+1) (0,+2) in (x, zeta), then (-2,0) (-1,0) (+1,0) (+2,0)
//  (-1,-1) (+1,-1) (-1,+1) (+1,+1) in (y, zeta)), B and the free-surface term
//==========================================================================
__global__ void KCzAssembleC(CzCoef k, const int *__restrict__ rowptr, const double *__restrict__ H,
                             const double *__restrict__ S, const double *__restrict__ C,
                             const double *__restrict__ Qx, const double *__restrict__ Qy,
                             const double *__restrict__ W, double *A, double *B, double *react)
{
	const int rx = k.nx - 4, ry = k.ny - 4, rz = k.nz - 4;
	const int nr = rx * ry * rz;
	const int sz = k.nx * k.ny;
	const double dx = k.dx, dy = k.dy, dzeta = k.dzeta, As = k.As, Df = k.Df;
	const bool limited = k.cI.limited != 0;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + (t / rx) % ry, kz = 2 + t / (rx * ry);
		auto Cc = [&](int i, int j, int q) { return C[I3(k, i, j, q)]; };
		auto Hh = [&](int i, int j) { return H[I2(k, i, j)]; };
		auto Ss = [&](int i, int j) { return S[I2(k, i, j)]; };
		const bool wallXmin = (ix == 2) && k.wall[0];
		const bool wallXmax = (ix == k.nx - 3) && k.wall[1];
		const bool wallYmin = (jy == 2) && k.wall[2];
		const bool wallYmax = (jy == k.ny - 3) && k.wall[3];
		const double hoo = Hh(ix, jy);
		const double hpo = Hh(ix + 1, jy), hPo = Hh(ix + 2, jy), hmo = Hh(ix - 1, jy), hMo = Hh(ix - 2, jy);
		const double spo = Ss(ix + 1, jy), sPo = Ss(ix + 2, jy), smo = Ss(ix - 1, jy), sMo = Ss(ix - 2, jy);
		const double soo = Ss(ix, jy);
		const double hL = 0.5 * (hoo + hmo), hR = 0.5 * (hoo + hpo);
		const double hx0 = (hMo - 8.0 * hmo + 8.0 * hpo - hPo) / (12.0 * dx);
		const double sx0 = (sMo - 8.0 * smo + 8.0 * spo - sPo) / (12.0 * dx);
		const double hxL = (hMo - 27.0 * hmo + 27.0 * hoo - hpo) / (24.0 * dx);
		const double sxL = (sMo - 27.0 * smo + 27.0 * soo - spo) / (24.0 * dx);
		const double hxR = (hmo - 27.0 * hoo + 27.0 * hpo - hPo) / (24.0 * dx);
		const double sxR = (smo - 27.0 * soo + 27.0 * spo - sPo) / (24.0 * dx);
		const double hoP = Hh(ix, jy + 2), hop = Hh(ix, jy + 1), hom = Hh(ix, jy - 1), hoM = Hh(ix, jy - 2);
		const double soP = Ss(ix, jy + 2), sop = Ss(ix, jy + 1), som = Ss(ix, jy - 1), soM = Ss(ix, jy - 2);
		const double hS = 0.5 * (hoo + hom), hN = 0.5 * (hoo + hop);
		const double hy0 = (hoM - 8.0 * hom + 8.0 * hop - hoP) / (12.0 * dy);
		const double sy0 = (soM - 8.0 * som + 8.0 * sop - soP) / (12.0 * dy);
		const double hyS = (hoM - 27.0 * hom + 27.0 * hoo - hop) / (24.0 * dy);
		const double syS = (soM - 27.0 * som + 27.0 * soo - sop) / (24.0 * dy);
		const double hyN = (hom - 27.0 * hoo + 27.0 * hop - hoP) / (24.0 * dy);
		const double syN = (som - 27.0 * soo + 27.0 * sop - soP) / (24.0 * dy);

		const int irow = I3(k, ix, jy, kz);
		const double zeta = dzeta * (-1.5 + (double)kz);
		const bool bottom = (kz == 2), top = (kz == k.nz - 3);
		double xz[5][5], yz[5][3];
		for(int a = 0; a < 5; ++a)
		{
			for(int b = 0; b < 5; ++b) xz[a][b] = 0.0;
			for(int b = 0; b < 3; ++b) yz[a][b] = 0.0;
		}
		double src = 0.0, rct = 0.0;
		auto X = [&](int di, int dk, double v) { xz[di + 2][dk + 2] += v; };
		auto Y = [&](int dj, int dk, double v) { if(dj == 0) xz[2][dk + 2] += v; else yz[dj + 2][dk + 1] += v; };
		//  advection: each face adds -F (c_f - c_P), F its outward volume flux
		{
			const double QL = Qx[irow], QR = Qx[irow + 1];
			const double fL[4] = {Cc(ix - 2, jy, kz), Cc(ix - 1, jy, kz), Cc(ix, jy, kz), Cc(ix + 1, jy, kz)};
			const double fR[4] = {Cc(ix - 1, jy, kz), Cc(ix, jy, kz), Cc(ix + 1, jy, kz), Cc(ix + 2, jy, kz)};
			double wL[4], wR[4];
			const double kL = 0, kR = 0;
			FaceWeights(k.cI, fL, QL, limited ? 2 : -1, wL);
			FaceWeights(k.cI, fR, QR, limited ? 1 : -1, wR);
			for(int q = 0; q < 4; ++q)
			{
				X(q - 2, 0, +QL * wL[q] / dx);
				X(q - 1, 0, -QR * wR[q] / dx);
			}
			src += (QL * kL - QR * kR) / dx;
		}
		{
			const double QS = Qy[irow], QN = Qy[irow + k.nx];
			const double fS[4] = {Cc(ix, jy - 2, kz), Cc(ix, jy - 1, kz), Cc(ix, jy, kz), Cc(ix, jy + 1, kz)};
			const double fN[4] = {Cc(ix, jy - 1, kz), Cc(ix, jy, kz), Cc(ix, jy + 1, kz), Cc(ix, jy + 2, kz)};
			double wS[4], wN[4];
			const double kS = 0, kN = 0;
			FaceWeights(k.cI, fS, QS, limited ? 2 : -1, wS);
			FaceWeights(k.cI, fN, QN, limited ? 1 : -1, wN);
			for(int q = 0; q < 4; ++q)
			{
				Y(q - 2, 0, +QS * wS[q] / dy);
				Y(q - 1, 0, -QN * wN[q] / dy);
			}
			src += (QS * kS - QN * kN) / dy;
		}
		{
			const double WB = W[irow], WT = W[irow + sz];
			if(!bottom)
			{
				const double fB[4] = {Cc(ix, jy, kz - 2), Cc(ix, jy, kz - 1), Cc(ix, jy, kz), Cc(ix, jy, kz + 1)};
				double wB[4];
				const double kB_ = 0;
				FaceWeights(k.cI, fB, WB, limited ? 2 : -1, wB);
				for(int q = 0; q < 4; ++q) X(0, q - 2, +WB * wB[q] / dzeta);
				src += WB * kB_ / dzeta;
			}
			if(!top)
			{
				const double fT[4] = {Cc(ix, jy, kz - 1), Cc(ix, jy, kz), Cc(ix, jy, kz + 1), Cc(ix, jy, kz + 2)};
				double wT[4];
				const double kT = 0;
				FaceWeights(k.cI, fT, WT, limited ? 1 : -1, wT);
				for(int q = 0; q < 4; ++q) X(0, q - 1, -WT * wT[q] / dzeta);
				src -= WT * kT / dzeta;
			}
			else
				rct += WT / dzeta;
		}
		//  diffusion through the x faces
		const double Coo = Cc(ix, jy, kz);
		{
			const double DL = Df * Diff(k, 0.5 * (Cc(ix - 1, jy, kz) + Coo));
			const double DR = Df * Diff(k, 0.5 * (Coo + Cc(ix + 1, jy, kz)));
			const double AL = (hxL * zeta + sxL) / hL;
			const double AR = (hxR * zeta + sxR) / hR;
			const double aL = wallXmin ? 0.0 : hL * DL / dx, aR = wallXmax ? 0.0 : hR * DR / dx;
			X(-1, 0, +aL / dx);
			X(0, 0, -aL / dx);
			X(-1, 1, +aL * AL / (4.0 * dzeta)); X(0, 1, +aL * AL / (4.0 * dzeta));
			X(-1, -1, -aL * AL / (4.0 * dzeta)); X(0, -1, -aL * AL / (4.0 * dzeta));
			X(1, 0, +aR / dx);
			X(0, 0, -aR / dx);
			X(0, 1, -aR * AR / (4.0 * dzeta)); X(1, 1, -aR * AR / (4.0 * dzeta));
			X(0, -1, +aR * AR / (4.0 * dzeta)); X(1, -1, +aR * AR / (4.0 * dzeta));
		}
		{
			const double DS = Df * Diff(k, 0.5 * (Cc(ix, jy - 1, kz) + Coo));
			const double DN = Df * Diff(k, 0.5 * (Coo + Cc(ix, jy + 1, kz)));
			const double AS = (hyS * zeta + syS) / hS;
			const double AN = (hyN * zeta + syN) / hN;
			const double aS = wallYmin ? 0.0 : hS * DS / dy, aN = wallYmax ? 0.0 : hN * DN / dy;
			Y(-1, 0, +aS / dy);
			Y(0, 0, -aS / dy);
			Y(-1, 1, +aS * AS / (4.0 * dzeta)); Y(0, 1, +aS * AS / (4.0 * dzeta));
			Y(-1, -1, -aS * AS / (4.0 * dzeta)); Y(0, -1, -aS * AS / (4.0 * dzeta));
			Y(1, 0, +aN / dy);
			Y(0, 0, -aN / dy);
			Y(0, 1, -aN * AN / (4.0 * dzeta)); Y(1, 1, -aN * AN / (4.0 * dzeta));
			Y(0, -1, +aN * AN / (4.0 * dzeta)); Y(1, -1, +aN * AN / (4.0 * dzeta));
		}
		//  diffusion through the interior zeta faces
		for(int side = 0; side < 2; ++side)
		{
			if(side == 0 && bottom) continue;
			if(side == 1 && top) continue;
			const int k0 = (side == 0) ? kz - 1 : kz;
			const double zf = zeta + (side == 0 ? -0.5 : 0.5) * dzeta;
			const double Dz = Df * Diff(k, 0.5 * (Cc(ix, jy, k0) + Cc(ix, jy, k0 + 1)));
			const double hA = hx0 * zf + sx0;
			const double hAy = hy0 * zf + sy0;
			const double g = (side == 1) ? +1.0 : -1.0;
			const double kzz = g * Dz * (As / hoo + (hA * hA + hAy * hAy) / hoo) / (dzeta * dzeta);
			X(0, k0 + 1 - kz, +kzz);
			X(0, k0 - kz, -kzz);
			const double kx = -g * Dz * hA / (4.0 * dx) / dzeta;
			X(1, k0 - kz, +kx); X(1, k0 + 1 - kz, +kx);
			X(-1, k0 - kz, -kx); X(-1, k0 + 1 - kz, -kx);
			const double ky = -g * Dz * hAy / (4.0 * dy) / dzeta;
			Y(1, k0 - kz, +ky); Y(1, k0 + 1 - kz, +ky);
			Y(-1, k0 - kz, -ky); Y(-1, k0 + 1 - kz, -ky);
		}
		//  the row: c_t = -A c - B with A = -R/h, the diagonal minus the sum
		//  of the rest plus the free-surface term
		const double rh = 1.0 / hoo;
		double offsum = 0.0;
		double *a = A + rowptr[irow];
		int q = 1;
		auto put = [&](double v) { a[q++] = -v * rh; offsum += -v * rh; };
		put(xz[2][0]); put(xz[1][1]); put(xz[2][1]); put(xz[3][1]);
		put(xz[0][2]); put(xz[1][2]); put(xz[3][2]); put(xz[4][2]);
		put(xz[1][3]); put(xz[2][3]); put(xz[3][3]); put(xz[2][4]);
		put(yz[0][1]); put(yz[1][1]); put(yz[3][1]); put(yz[4][1]);
		put(yz[1][0]); put(yz[3][0]); put(yz[1][2]); put(yz[3][2]);
		const double r = -rct * rh;
		react[irow] = r;
		a[0] = -offsum + r;
		B[irow] = -src * rh - 0.0;
	}
}

//  SetBoundaryCondition (:613-700), the zeta ghosts of every real column:
//  the right-hand sides that give the conormal flux its value at the
//  substrate (zero) and at the free surface (the solvent leaving, without
//  its solute); atEnd: with the evaporation of the end state
__global__ void KCzBcC(CzCoef k, const double *__restrict__ H, const double *__restrict__ S,
                       const double *__restrict__ C, const double *__restrict__ W, int atEnd, double dt, double *Rhs)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4);
	const double dzeta = k.dzeta, dx = k.dx, dy = k.dy, As = k.As, Df = k.Df;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + t / rx;
		auto Cc = [&](int i, int j, int q) { return C[I3(k, i, j, q)]; };
		auto Hh = [&](int i, int j) { return H[I2(k, i, j)]; };
		auto Ss = [&](int i, int j) { return S[I2(k, i, j)]; };
		const double hh = Hh(ix, jy);
		const double hx0 = (Hh(ix - 2, jy) - 8.0 * Hh(ix - 1, jy) + 8.0 * Hh(ix + 1, jy) - Hh(ix + 2, jy)) / (12.0 * dx);
		const double sx0 = (Ss(ix - 2, jy) - 8.0 * Ss(ix - 1, jy) + 8.0 * Ss(ix + 1, jy) - Ss(ix + 2, jy)) / (12.0 * dx);
		const double hy0 = (Hh(ix, jy - 2) - 8.0 * Hh(ix, jy - 1) + 8.0 * Hh(ix, jy + 1) - Hh(ix, jy + 2)) / (12.0 * dy);
		const double sy0 = (Ss(ix, jy - 2) - 8.0 * Ss(ix, jy - 1) + 8.0 * Ss(ix, jy + 1) - Ss(ix, jy + 2)) / (12.0 * dy);
		const double gB = 0.0;
		{
			const int q = 2;
			const double cb = 0.5 * (Cc(ix, jy, q - 1) + Cc(ix, jy, q));
			const double D = Df * Diff(k, cb);
			const double cx = (Cc(ix + 1, jy, q) - Cc(ix - 1, jy, q)) / (2.0 * dx);
			const double cy = (Cc(ix, jy + 1, q) - Cc(ix, jy - 1, q)) / (2.0 * dy);
			const double hA = sx0, hAy = sy0;
			const double cz = hh * (gB / D + hA * cx + hAy * cy) / (As + hA * hA + hAy * hAy);
			Rhs[I3(k, ix, jy, 0)] = -3.0 * dzeta * cz;
			Rhs[I3(k, ix, jy, 1)] = -dzeta * cz;
		}
		{
			const int q = k.nz - 3;
			const double cs = 0.5 * (Cc(ix, jy, q) + Cc(ix, jy, q + 1));
			const double D = Df * Diff(k, cs);
			const double cx = (Cc(ix + 1, jy, q) - Cc(ix - 1, jy, q)) / (2.0 * dx);
			const double cy = (Cc(ix, jy + 1, q) - Cc(ix, jy - 1, q)) / (2.0 * dy);
			const double hA = hx0 + sx0, hAy = hy0 + sy0;
			double WT = W[I3(k, ix, jy, k.nz - 2)];
			if(atEnd)
			{
				WT = k.onEvap ? EvapCol(k, H, C, ix, jy) : 0.0;
				double cm = 0.0;
				for(int kk = 2; kk < k.nz - 2; ++kk) cm += Cc(ix, jy, kk);
				cm /= (double)(k.nz - 4);
				WT = SolventLimitCz(WT, hh, cm, dt);
			}
			const double G = WT * cs;
			const double cz = hh * (G / D + hA * cx + hAy * cy) / (As + hA * hA + hAy * hAy);
			const double grad = dzeta * cz;
			Rhs[I3(k, ix, jy, k.nz - 2)] = grad;
			Rhs[I3(k, ix, jy, k.nz - 1)] = 3.0 * grad;
		}
	}
}

//  ApplyBoundaryRows (:992-1005): each ghost row x_r = Rhs_r + x_partner; the
//  zeta ghosts of the real columns first, then the y ghosts of the real
//  columns, then the x ghosts (a corner reads a y ghost, an edge ghost a
//  zeta ghost), where the reference's sweeps in row order end up
__global__ void KCzApplyZ(CzCoef k, const double *__restrict__ Rhs, double *x)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr * 4; t += gridDim.x * blockDim.x)
	{
		const int c = t % nr, g = t / nr;
		const int ix = 2 + c % rx, jy = 2 + c / rx;
		const int kz = g < 2 ? g : k.nz - 4 + g;
		const int p = (kz == 0) ? 3 : (kz == 1) ? 2 : (kz == k.nz - 2) ? k.nz - 3 : k.nz - 4;
		const int r = I3(k, ix, jy, kz);
		double sum = Rhs[r];
		sum -= -1.0 * x[I3(k, ix, jy, p)];
		x[r] = sum / 1.0;
	}
}
__global__ void KCzApplyY(CzCoef k, const double *__restrict__ Rhs, double *x)
{
	const int rx = k.nx - 4, n = rx * 4 * k.nz;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, g = (t / rx) % 4, kz = t / (rx * 4);
		const int jy = g < 2 ? g : k.ny - 4 + g;
		int p;
		if(k.perY) p = (jy == 0) ? k.ny - 4 : (jy == 1) ? k.ny - 3 : (jy == k.ny - 2) ? 2 : 3;
		else p = (jy == 0) ? 3 : (jy == 1) ? 2 : (jy == k.ny - 2) ? k.ny - 3 : k.ny - 4;
		const int r = I3(k, ix, jy, kz);
		double sum = Rhs[r];
		sum -= -1.0 * x[I3(k, ix, p, kz)];
		x[r] = sum / 1.0;
	}
}
__global__ void KCzApplyX(CzCoef k, const double *__restrict__ Rhs, double *x)
{
	const int n = k.ny * 4 * k.nz;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
	{
		const int jy = t % k.ny, g = (t / k.ny) % 4, kz = t / (k.ny * 4);
		const int ix = g < 2 ? g : k.nx - 4 + g;
		int p;
		if(k.perX) p = (ix == 0) ? k.nx - 4 : (ix == 1) ? k.nx - 3 : (ix == k.nx - 2) ? 2 : 3;
		else p = (ix == 0) ? 3 : (ix == 1) ? 2 : (ix == k.nx - 2) ? k.nx - 3 : k.nx - 4;
		const int r = I3(k, ix, jy, kz);
		double sum = Rhs[r];
		sum -= -1.0 * x[I3(k, p, jy, kz)];
		x[r] = sum / 1.0;
	}
}

//  ExplicitPart (:894-909): A x as sum_j a_ij (x_j - x_i) + r_i x_i on the
//  real rows, zero on the ghost rows
__global__ void KCzExplicit(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                            const unsigned char *__restrict__ bc, const double *__restrict__ A,
                            const double *__restrict__ react, const double *__restrict__ x, double *Ax)
{
	for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
	{
		if(bc[r]) { Ax[r] = 0.0; continue; }
		const double xr = x[r];
		double s = react[r] * xr;
		const int ed = rowptr[r + 1];
		for(int q = rowptr[r] + 1; q < ed; ++q) s += A[q] * (x[col[q]] - xr);
		Ax[r] = s;
	}
}

//  the right-hand side of the change over a step, -dt (A c_old + B) on the
//  real rows (0 on the ghost rows), and whether any of it is not zero
__global__ void KCzRhsC(int n, const unsigned char *__restrict__ bc, const double *__restrict__ Ax,
                        const double *__restrict__ B, double dt, double *rhs, int *any)
{
	int mine = 0;
	for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
	{
		double v = 0.0;
		if(!bc[r]) { v = -dt * (Ax[r] + B[r]); if(v != 0.0) mine = 1; }
		rhs[r] = v;
	}
	if(__any_sync(0xffffffffu, mine) && (threadIdx.x & 31) == 0) atomicOr(any, 1);
}

} // namespace

namespace {

//==========================================================================
//  Reductions (fixed order: a grid of kRedBlocks blocks, each a 256-thread
//  tree, the partials folded by one block)
//==========================================================================
constexpr int kRedBlocks = 296;

//  Aitken weights of the coupling passes (:309-320): sum rPrev (r - rPrev)
//  and sum (r - rPrev)^2 over every row
__global__ void __launch_bounds__(256) KCzAitken(long long n, const double *__restrict__ r,
                                                 const double *__restrict__ rp, double *part)
{
	__shared__ double sh[2 * kRT];
	double a[2] = {0.0, 0.0};
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		const double d = r[i] - rp[i];
		a[0] += rp[i] * d;
		a[1] += d * d;
	}
	BlockTree<2>(a, sh);
	if(threadIdx.x == 0) { part[blockIdx.x] = a[0]; part[kRedBlocks + blockIdx.x] = a[1]; }
}

//  the solute the solve's residual leaves (SolveStage, :845-866): sum over
//  the real cells of h (-dt (A c_theta + B) - d) and of h (1 + theta dt react)
__global__ void __launch_bounds__(256) KCzAlpha(CzCoef k, const double *__restrict__ H, const double *__restrict__ Ac,
                                                const double *__restrict__ B, const double *__restrict__ d,
                                                const double *__restrict__ react, double dt, double theta, double *part)
{
	__shared__ double sh[2 * kRT];
	const int rx = k.nx - 4, ry = k.ny - 4, nr = rx * ry * (k.nz - 4);
	double a[2] = {0.0, 0.0};
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + (t / rx) % ry, kz = 2 + t / (rx * ry);
		const int r = I3(k, ix, jy, kz);
		const double h = H[I2(k, ix, jy)];
		a[0] += h * (-dt * (Ac[r] + B[r]) - d[r]);
		a[1] += h * (1.0 + theta * dt * react[r]);
	}
	BlockTree<2>(a, sh);
	if(threadIdx.x == 0) { part[blockIdx.x] = a[0]; part[kRedBlocks + blockIdx.x] = a[1]; }
}

__global__ void __launch_bounds__(256) KCzFold2(const double *__restrict__ part, double *out)
{
	__shared__ double sh[2 * kRT];
	double a[2] = {0.0, 0.0};
	for(int j = threadIdx.x; j < kRedBlocks; j += blockDim.x)
	{
		a[0] += part[j];
		a[1] += part[kRedBlocks + j];
	}
	BlockTree<2>(a, sh);
	if(threadIdx.x == 0) { out[0] = a[0]; out[1] = a[1]; }
}

__global__ void KCzAbsMax(long long n, const double *__restrict__ x, unsigned long long *out)
{
	double m = 0.0;
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		m = fmax(m, fabs(x[i]));
	MaxAbsInto(out, m);
}

//  LocalTruncationCriterion (ImplicitSolver.cpp:271-307): max |E_k|
__global__ void KCzLte(int n, const double *__restrict__ hp, const double *__restrict__ ho, const double *__restrict__ hm,
                       double dt0, double dt, double wfloor, unsigned long long *out)
{
	double m = 0.0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		double w = fabs(ho[i]);
		if(w < wfloor) w = wfloor;
		const double denom = (dt0 + dt) * w;
		const double e = (fabs(denom) <= 2.2250738585072014e-308)
		    ? 0.0 : 2.0 * (dt / dt0) * (dt0 * hp[i] + dt * hm[i] - (dt0 + dt) * ho[i]) / denom;
		m = fmax(m, fabs(e));
	}
	MaxAbsInto(out, m);
}

//==========================================================================
//  Element-wise steps of the passes
//==========================================================================
//  (a + b) * 0.5
__global__ void KCzMid(long long n, const double *__restrict__ a, const double *__restrict__ b, double *out)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		double v = a[i];
		v += b[i];
		out[i] = v * 0.5;
	}
}

//  MidpointConc (:1979-1986): x + r (x - prev)
__global__ void KCzExtrap(long long n, const double *__restrict__ x, const double *__restrict__ prev, double r, double *out)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		out[i] = x[i] + r * (x[i] - prev[i]);
}

//  the coupling residual ((c0 + c) * 0.5) - cm
__global__ void KCzCoupleRes(long long n, const double *__restrict__ c0, const double *__restrict__ c,
                             const double *__restrict__ cm, double *r)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		double v = c0[i];
		v += c[i];
		v *= 0.5;
		r[i] = v - cm[i];
	}
}

//  x[i] += w y[i]
__global__ void KCzAxpy(long long n, double w, const double *__restrict__ y, double *x)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		x[i] += w * y[i];
}

//  x[i] += s
__global__ void KCzShift(long long n, double s, double *x)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		x[i] += s;
}

//  d <- (old + d) with the boundary rows applied, less old (two kernels
//  around ApplyBoundaryRows): here out = a + b, and out = a - b
__global__ void KCzAdd(long long n, const double *__restrict__ a, const double *__restrict__ b, double *out)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		double v = a[i];
		v += b[i];
		out[i] = v;
	}
}
__global__ void KCzSub(long long n, const double *__restrict__ a, const double *__restrict__ b, double *out)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		double v = a[i];
		v -= b[i];
		out[i] = v;
	}
}

//  c_theta = d theta + old
__global__ void KCzTheta(long long n, const double *__restrict__ d, const double *__restrict__ old, double theta, double *ct)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		double v = d[i];
		v *= theta;
		v += old[i];
		ct[i] = v;
	}
}

//  the largest change between two passes of the limiter and over the step
//  (SettleLimiter, :949-979)
__global__ void KCzLimMax(long long n, const double *__restrict__ nw, const double *__restrict__ prev,
                          const double *__restrict__ old, unsigned long long *out)
{
	double a = 0.0, b = 0.0;
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
	{
		a = fmax(a, fabs(nw[i] - prev[i]));
		b = fmax(b, fabs(nw[i] - old[i]));
	}
	MaxAbsInto(out, a);
	MaxAbsInto(out + 1, b);
}

//==========================================================================
//  RedistributeExcess (CZ_HeightEquation_2D.cpp:403-447): per real column,
//  c above 1 passed down, what reaches the substrate back up
//==========================================================================
__global__ void KCzExcess(CzCoef k, double *c)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4);
	const int kb = 2, kt = k.nz - 3;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + t / rx;
		auto at = [&](int q) -> double & { return c[I3(k, ix, jy, q)]; };
		bool any = false;
		for(int q = kb; q <= kt; ++q) if(at(q) > 1.0) { any = true; break; }
		if(!any) continue;
		for(int q = kt; q > kb; --q)
		{
			double &ck = at(q);
			if(ck > 1.0) { const double e = ck - 1.0; ck = 1.0; at(q - 1) += e; }
		}
		double &cb = at(kb);
		if(cb > 1.0)
		{
			double e = cb - 1.0;
			cb = 1.0;
			for(int q = kb + 1; q <= kt && e > 0.0; ++q)
			{
				double &ck = at(q);
				const double take = fmin(e, 1.0 - ck);
				if(take > 0.0) { ck += take; e -= take; }
			}
			if(e > 0.0)
				for(int q = kb; q <= kt; ++q) at(q) += e / (double)(kt - kb + 1);
		}
	}
}

//  RedistributeDeficit (:449-570), the columns: whether a real cell is
//  below 0 (flag[0]); then within each column its cells below 0 from its
//  cells above, a column with less than no solute in all left with its mean
//  (flag[1]: such a column, whose lack is taken from the columns around)
__global__ void KCzDeficitAny(CzCoef k, const double *__restrict__ c, int *flag)
{
	const int rx = k.nx - 4, ry = k.ny - 4, nr = rx * ry * (k.nz - 4);
	int mine = 0;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + (t / rx) % ry, kz = 2 + t / (rx * ry);
		if(c[I3(k, ix, jy, kz)] < 0.0) mine = 1;
	}
	if(__any_sync(0xffffffffu, mine) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}
__global__ void KCzDeficitCol(CzCoef k, double *c, int *flag)
{
	const int rx = k.nx - 4, nr = rx * (k.ny - 4);
	const int kb = 2, kt = k.nz - 3;
	const double nLay = (double)(kt - kb + 1);
	int mine = 0;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % rx, jy = 2 + t / rx;
		auto at = [&](int q) -> double & { return c[I3(k, ix, jy, q)]; };
		double def = 0.0, pos = 0.0;
		for(int q = kb; q <= kt; ++q)
		{
			const double ck = at(q);
			if(ck < 0.0) def -= ck; else pos += ck;
		}
		if(def == 0.0) continue;
		if(pos >= def)
		{
			const double f = def / pos;
			for(int q = kb; q <= kt; ++q)
			{
				double &ck = at(q);
				ck = (ck < 0.0) ? 0.0 : ck - f * ck;
			}
		}
		else
		{
			const double m = (pos - def) / nLay;
			for(int q = kb; q <= kt; ++q) at(q) = m;
			mine = 1;
		}
	}
	if(__any_sync(0xffffffffu, mine) && (threadIdx.x & 31) == 0) atomicOr(flag + 1, 1);
}

} // namespace

//  the correctly rounded exp of yz_exp.h, element by element (its test)
__global__ void KCrExp(long long n, const double *__restrict__ x, double *y)
{
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		y[i] = crexp::Exp(x[i]);
}

//==========================================================================
//  Host side
//==========================================================================
namespace {

//  the sorted mirror of a pattern (CRS_Matrix::BuildSortPermutation,
//  CRS_Matrix.cpp:360-384)
void SortedMirror(const std::vector<int> &rowptr, const std::vector<int> &col, std::vector<int> &scol,
                  std::vector<int> &ssrc)
{
	const int n = (int)rowptr.size() - 1;
	scol.assign(col.size(), 0);
	ssrc.assign(col.size(), 0);
	std::vector<std::pair<int, int>> tmp;
	for(int i = 0; i < n; ++i)
	{
		const int st = rowptr[(size_t)i], ed = rowptr[(size_t)i + 1];
		tmp.clear();
		for(int q = st; q < ed; ++q) tmp.push_back({col[(size_t)q], q});
		std::sort(tmp.begin(), tmp.end());
		for(int q = st; q < ed; ++q)
		{
			scol[(size_t)q] = tmp[(size_t)(q - st)].first;
			ssrc[(size_t)q] = tmp[(size_t)(q - st)].second;
		}
	}
}

int GhostPartner(int i, int n, bool per)
{
	if(per) return (i == 0) ? n - 4 : (i == 1) ? n - 3 : (i == n - 2) ? 2 : 3;
	return (i == 0) ? 3 : (i == 1) ? 2 : (i == n - 2) ? n - 3 : n - 4;
}

bool IsWallKind(int t) { return t == kBcSym || t == kBcPin; }

} // namespace

void CheckCzParams(const yz_cz_params &p)
{
	if(p.ny < 8 || p.nx < 8 || p.nz < 7)
		throw UsageError("cz: nx, ny >= 8 and nz >= 7 (the ghost layers included); the 1-D film (ny = 1) is not "
		                 "on this path");
	//  the edge kinds the reference's CZ model implements
	//  (CheckParameters.cpp:340-353 refuses the others for it)
	for(int e = 0; e < 4; ++e)
		if(p.bc[e] != kBcSym && p.bc[e] != kBcPer)
			throw UsageError("cz: the CZ model implements only Symmetry and Periodic boundaries");
	if((p.bc[0] == kBcPer) != (p.bc[1] == kBcPer) || (p.bc[2] == kBcPer) != (p.bc[3] == kBcPer))
		throw UsageError("cz: a Periodic edge needs the opposite edge Periodic too");
	if(p.c_scheme < YZ_SCHEME_UPWIND1 || p.c_scheme > YZ_SCHEME_VANLEER) throw UsageError("cz: unknown scheme");
	if(!(p.dx > 0 && p.dy > 0 && p.dzeta > 0 && p.dt > 0)) throw UsageError("cz: dx, dy, dzeta and dt must be > 0");
	if(!(p.theta_h > 0.0) || !(p.theta_c > 0.0))
		throw UsageError("cz: theta_h and theta_c must be > 0 (the explicit scheme is not on this path)");
}

//  the patterns of the film's and the concentration's matrices in the
//  reference's storage order: the order in which SetMatrixA first writes the
//  columns of a row (CZ_HeightEquation_2D.cpp:750-1081,
//  CZ_ConcEquation_2D.cpp:301-700), the diagonal first
void BuildCzPatterns(const yz_cz_params &p, std::vector<int> &rowptrH, std::vector<int> &colH, std::vector<int> &bcH,
                     std::vector<int> &rowptrC, std::vector<int> &colC, std::vector<int> &bcC)
{
	const int nx = p.nx, ny = p.ny, nz = p.nz;
	const bool perX = p.bc[0] == kBcPer && p.bc[1] == kBcPer, perY = p.bc[2] == kBcPer && p.bc[3] == kBcPer;
	auto real2 = [&](int ix, int jy) { return ix >= 2 && ix < nx - 2 && jy >= 2 && jy < ny - 2; };
	rowptrH.assign(1, 0);
	colH.clear();
	bcH.assign((size_t)nx * ny, 0);
	for(int jy = 0; jy < ny; ++jy)
		for(int ix = 0; ix < nx; ++ix)
		{
			const int r = jy * nx + ix;
			auto C2 = [&](int i, int j) { colH.push_back(j * nx + i); };
			if(real2(ix, jy))
			{
				C2(ix, jy);
				C2(ix - 2, jy); C2(ix - 1, jy); C2(ix + 1, jy); C2(ix + 2, jy);
				C2(ix, jy - 2); C2(ix, jy - 1); C2(ix, jy + 1); C2(ix, jy + 2);
				C2(ix - 1, jy - 1); C2(ix - 1, jy + 1); C2(ix + 1, jy - 1); C2(ix + 1, jy + 1);
			}
			else
			{
				bcH[(size_t)r] = 1;
				C2(ix, jy);
				if(ix < 2 || ix >= nx - 2) C2(GhostPartner(ix, nx, perX), jy);
				else C2(ix, GhostPartner(jy, ny, perY));
			}
			rowptrH.push_back((int)colH.size());
		}
	rowptrC.assign(1, 0);
	colC.clear();
	bcC.assign((size_t)nx * ny * nz, 0);
	for(int kz = 0; kz < nz; ++kz)
		for(int jy = 0; jy < ny; ++jy)
			for(int ix = 0; ix < nx; ++ix)
			{
				const int r = (kz * ny + jy) * nx + ix;
				auto C3 = [&](int i, int j, int q) { colC.push_back((q * ny + j) * nx + i); };
				const bool rc = real2(ix, jy);
				if(rc && kz >= 2 && kz < nz - 2)
				{
					C3(ix, jy, kz);
					C3(ix, jy, kz - 2); C3(ix - 1, jy, kz - 1); C3(ix, jy, kz - 1); C3(ix + 1, jy, kz - 1);
					C3(ix - 2, jy, kz); C3(ix - 1, jy, kz); C3(ix + 1, jy, kz); C3(ix + 2, jy, kz);
					C3(ix - 1, jy, kz + 1); C3(ix, jy, kz + 1); C3(ix + 1, jy, kz + 1); C3(ix, jy, kz + 2);
					C3(ix, jy - 2, kz); C3(ix, jy - 1, kz); C3(ix, jy + 1, kz); C3(ix, jy + 2, kz);
					C3(ix, jy - 1, kz - 1); C3(ix, jy + 1, kz - 1); C3(ix, jy - 1, kz + 1); C3(ix, jy + 1, kz + 1);
				}
				else
				{
					bcC[(size_t)r] = 1;
					C3(ix, jy, kz);
					if(rc)
						C3(ix, jy, (kz == 0) ? 3 : (kz == 1) ? 2 : (kz == nz - 2) ? nz - 3 : nz - 4);
					else if(ix < 2 || ix >= nx - 2)
						C3(GhostPartner(ix, nx, perX), jy, kz);
					else
						C3(ix, GhostPartner(jy, ny, perY), kz);
				}
				rowptrC.push_back((int)colC.size());
			}
}


CzStep::CzStep(int device, const yz_cz_params &p, const double *xc, const double *xf, const double *yc,
               const double *yf, const double *h, const double *s, const double *c)
    : _device(device), _p(p)
{
	CheckCzParams(p);
	YZ_CUDA(cudaSetDevice(device));
	YZ_CUDA(cudaStreamCreateWithFlags(&_st, cudaStreamNonBlocking));
	const int nx = p.nx, ny = p.ny, nz = p.nz;
	_n2 = nx * ny;
	_n3 = nx * ny * nz;

	CzCoef &k = _k;
	std::memset(&k, 0, sizeof(k));
	k.nx = nx; k.ny = ny; k.nz = nz;
	k.perX = (p.bc[0] == kBcPer && p.bc[1] == kBcPer) ? 1 : 0;
	k.perY = (p.bc[2] == kBcPer && p.bc[3] == kBcPer) ? 1 : 0;
	k.perXv = (p.bc[0] == kBcPer) ? 1 : 0;
	k.perYv = (p.bc[2] == kBcPer) ? 1 : 0;
	for(int e = 0; e < 4; ++e) k.wall[e] = IsWallKind(p.bc[e]) ? 1 : 0;
	k.onL = p.on_lap; k.onSC = p.on_sc; k.onVG = p.on_vg; k.onHG = p.on_hg; k.onCF = p.on_cf; k.onEvap = p.on_evap;
	k.dx = p.dx; k.dy = p.dy; k.dzeta = p.dzeta;
	k.rdx = 1.0 / p.dx; k.rdx2 = k.rdx * k.rdx; k.rdx4 = k.rdx2 * k.rdx2;
	k.rdy = 1.0 / p.dy; k.rdy2 = k.rdy * k.rdy; k.rdy4 = k.rdy2 * k.rdy2;
	k.rdx2dy2 = k.rdx2 * k.rdy2;
	k.dx3 = std::pow(p.dx, 3.0);
	k.dy3 = std::pow(p.dy, 3.0);
	k.As = p.As; k.Ma = p.Ma; k.Bo = p.Bo; k.Pgx = p.Pgx; k.Pgy = p.Pgy; k.Sp = p.Sp; k.Df = p.Df; k.Ev = p.Ev;
	k.rot0 = p.rot_center[0]; k.rot1 = p.rot_center[1];
	k.diffC0 = p.diff_c0; k.diffBase = p.diff_base; k.diffExp = p.diff_exp;
	k.ev.viscC0 = p.visc_c0; k.ev.viscBase = p.visc_base; k.ev.viscExp = p.visc_exp;
	k.ev.sigC0 = p.sig_c0; k.ev.sigBase = p.sig_base; k.ev.sigCoef = p.sig_coef;
	k.ev.Ev = p.Ev;
	k.ev.evConc = p.ev_conc; k.ev.evSpatial = p.ev_spatial; k.ev.evHast = p.ev_hast;
	k.ev.evMr = p.ev_mr; k.ev.evMs = p.ev_ms; k.ev.evPowN = p.ev_pown; k.ev.evConcR = p.ev_concr;
	k.ev.evNegExp = p.ev_negexp; k.ev.evNegRmax = p.ev_negrmax; k.ev.evHast_h = p.ev_hast_h; k.ev.evDr = p.ev_dr;
	k.cI = MakeInterp(p.c_scheme);

	BuildCzPatterns(p, _rowptrH, _colH, _bcH, _rowptrC, _colC, _bcC);
	_nnzH = (int)_colH.size();
	_nnzC = (int)_colC.size();

	_solverH.reset(new Solver(device, _st));
	_solverC.reset(new Solver(device, _st));
	{
		std::vector<int> scol, ssrc;
		SortedMirror(_rowptrH, _colH, scol, ssrc);
		_solverH->SetPattern(_n2, _nnzH, _rowptrH.data(), scol.data(), ssrc.data());
		SortedMirror(_rowptrC, _colC, scol, ssrc);
		_solverC->SetPattern(_n3, _nnzC, _rowptrC.data(), scol.data(), ssrc.data());
	}
	_dRowptrH.upload(_rowptrH.data(), _rowptrH.size(), _st);
	_dColH.upload(_colH.data(), _colH.size(), _st);
	_dRowptrC.upload(_rowptrC.data(), _rowptrC.size(), _st);
	_dColC.upload(_colC.data(), _colC.size(), _st);
	{
		std::vector<unsigned char> b(_bcH.begin(), _bcH.end());
		_dBcH.upload(b.data(), b.size(), _st);
		std::vector<unsigned char> bc(_bcC.begin(), _bcC.end());
		_dBcC.upload(bc.data(), bc.size(), _st);
	}
	_xc.upload(xc, (size_t)nx, _st); _xf.upload(xf, (size_t)nx, _st);
	_yc.upload(yc, (size_t)ny, _st); _yf.upload(yf, (size_t)ny, _st);
	k.xc = _xc.get(); k.xf = _xf.get(); k.yc = _yc.get(); k.yf = _yf.get();

	const size_t n2 = (size_t)_n2, n3 = (size_t)_n3;
	for(DBuf<double> *b : {&_s, &_fH, &_tH, &_hOld2, &_hOld, &_hNew, &_B, &_Ax, &_rhs, &_colSrc, &_dtdh, &_hc,
	                       &_hMid})
	{
		b->reserve(n2);
		YZ_CUDA(cudaMemsetAsync(b->get(), 0, n2 * sizeof(double), _st));
	}
	for(int a = 0; a < 2; ++a)
		for(DBuf<double> *b : {&_D[a], &_sig[a], &_M[a], &_qCap[a], &_qExp[a], &_q[a]})
		{
			b->reserve(n2);
			YZ_CUDA(cudaMemsetAsync(b->get(), 0, n2 * sizeof(double), _st));
		}
	for(DBuf<double> *b : {&_fC, &_tC, &_cOld2, &_cOld, &_cNew, &_Bc, &_Rc, &_react, &_Axc, &_rhsc, &_d, &_ct,
	                       &_Qx, &_Qy, &_W, &_Ux, &_Uy, &_kOld2, &_kOld, &_kNew, &_ccPrev, &_ccPrevKeep, &_c0, &_cm,
	                       &_r, &_rPrev, &_mid, &_prev})
	{
		b->reserve(n3);
		YZ_CUDA(cudaMemsetAsync(b->get(), 0, n3 * sizeof(double), _st));
	}
	//  the matrices' ghost rows are constant ([1, -1]); the real rows are
	//  written by every assembly
	{
		std::vector<double> v((size_t)_nnzH, 0.0);
		for(int r = 0; r < _n2; ++r)
			if(_bcH[(size_t)r]) { v[(size_t)_rowptrH[(size_t)r]] = 1.0; v[(size_t)_rowptrH[(size_t)r] + 1] = -1.0; }
		_A.upload(v.data(), v.size(), _st);
		_IA.upload(v.data(), v.size(), _st);
		std::vector<double> w((size_t)_nnzC, 0.0);
		for(int r = 0; r < _n3; ++r)
			if(_bcC[(size_t)r]) { w[(size_t)_rowptrC[(size_t)r]] = 1.0; w[(size_t)_rowptrC[(size_t)r] + 1] = -1.0; }
		_Ac.upload(w.data(), w.size(), _st);
		_IAc.upload(w.data(), w.size(), _st);
	}
	_s.upload(s, n2, _st);
	for(DBuf<double> *b : {&_fH, &_tH, &_hOld2, &_hOld, &_hNew}) b->upload(h, n2, _st);
	for(DBuf<double> *b : {&_fC, &_tC, &_cOld2, &_cOld, &_cNew}) b->upload(c, n3, _st);
	_red.reserve(2 * kRedBlocks + 8);
	_max.reserve(4);
	_flag.reserve(4);
	_dt = p.dt;
	_dtOld = p.dt_old;
	_time = p.time;
	YZ_CUDA(cudaStreamSynchronize(_st));
}

CzStep::~CzStep()
{
	cudaSetDevice(_device);
	if(_st) cudaStreamSynchronize(_st);
	_solverH.reset();
	_solverC.reset();
	_learned.reset();
	if(_st) cudaStreamDestroy(_st);
}

void CzStep::Copy(double *dst, const double *src, size_t n)
{
	if(dst != src) YZ_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
}

double CzStep::AbsMax(const double *x, long long n)
{
	YZ_CUDA(cudaMemsetAsync(_max.get(), 0, sizeof(unsigned long long), _st));
	YZ_LAUNCH(KCzAbsMax, GridFor(n, kB), kB, 0, _st, n, x, _max.get());
	unsigned long long u = 0;
	YZ_CUDA(cudaMemcpyAsync(&u, _max.get(), sizeof(u), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	double v;
	std::memcpy(&v, &u, sizeof(v));
	return v;
}

void CzStep::ZeroFlag() { YZ_CUDA(cudaMemsetAsync(_flag.get(), 0, 4 * sizeof(int), _st)); }

bool CzStep::Flag()
{
	int f = 0;
	YZ_CUDA(cudaMemcpyAsync(&f, _flag.get(), sizeof(int), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	return f != 0;
}

//--------------------------------------------------------------------------
//  the film
//--------------------------------------------------------------------------
void CzStep::SetMatrixAH(const double *fH, const double *fC, double dt)
{
	const int nf = (_p.nx - 3) * (_p.ny - 4) + (_p.nx - 4) * (_p.ny - 3);
	YZ_LAUNCH(KCzFaces, GridFor(nf, kB), kB, 0, _st, _k, fH, _s.get(), fC, _D[0].get(), _sig[0].get(), _M[0].get(),
	          _qCap[0].get(), _qExp[0].get(), _D[1].get(), _sig[1].get(), _M[1].get(), _qCap[1].get(), _qExp[1].get());
	const int nr = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KCzAssembleH, GridFor(nr, kB), kB, 0, _st, _k, _dRowptrH.get(), fH, _s.get(), fC, _tH.get(), _tC.get(),
	          _D[0].get(), _sig[0].get(), _M[0].get(), _D[1].get(), _sig[1].get(), _M[1].get(), dt, _A.get(), _B.get(),
	          _colSrc.get());
}

//  SolveStage (CZ_HeightEquation_2D.cpp:1949-1963)
void CzStep::SolveStageH(const double *fH, const double *fC, double dt, int &iter, double &resid, int &ch)
{
	{
		YZ_PROF("h.assemble", _st);
		SetMatrixAH(fH, fC, dt);
	}
	const int g = GridFor(_n2, kB);
	{
		YZ_PROF("h.rhs", _st);
		YZ_LAUNCH(KCzMatVec, g, kB, 0, _st, _n2, _dRowptrH.get(), _dColH.get(), _A.get(), _hOld.get(), _Ax.get());
		YZ_LAUNCH(KCzMakeIA, g, kB, 0, _st, _n2, _dRowptrH.get(), _dBcH.get(), _A.get(), _IA.get(), _p.theta_h, dt);
		YZ_LAUNCH(KCzMakeRhsH, g, kB, 0, _st, _n2, _dBcH.get(), _hOld.get(), _Ax.get(), _B.get(), _p.theta_h, dt,
		          _rhs.get());
	}
	iter = 0;
	resid = 0;
	//  the learned preconditioner reads the stage's film as a feature, and is
	//  trained once the solves that collect its pairs are done
	if(_learned)
	{
		_solverH->SetAux(fH);
		if(!_learned->Trained() && _solverH->CollectLeft() == 0) TrainLearned();
	}
	{
		YZ_PROF("h.linsolve", _st);
		ch = _solverH->Solve(_p.h_lin, _IA.get(), _rhs.get(), _hNew.get(), iter, resid);
	}
	++_solves;
}

//  Solve (:1988-2020): the predictor with the coefficients of the start of
//  the step, then the corrector with h halfway and c extrapolated half a step
void CzStep::SolveH(double dt, int &iter, double &resid, int &ch)
{
	SolveStageH(_fH.get(), _fC.get(), dt, iter, resid, ch);
	if(ch != 0) return;
	const long long n2 = _n2, n3 = _n3;
	YZ_LAUNCH(KCzMid, GridFor(n2, kB), kB, 0, _st, n2, _hOld.get(), _hNew.get(), _fH.get());
	const bool extrapolate = _ccPrevSet;
	if(extrapolate)
		YZ_LAUNCH(KCzExtrap, GridFor(n3, kB), kB, 0, _st, n3, _cNew.get(), _ccPrev.get(), 0.5 * dt / _dtPrev, _fC.get());
	int it2 = 0;
	double r2 = 0;
	SolveStageH(_fH.get(), _fC.get(), dt, it2, r2, ch);
	iter += it2;
	resid = r2;
	Copy(_fH.get(), _hOld.get(), (size_t)_n2);
	if(extrapolate) Copy(_fC.get(), _cNew.get(), (size_t)_n3);
}

void CzStep::CopyGhostsH(double *h)
{
	YZ_LAUNCH(KCzGhostY, GridFor((_p.nx - 4) * 4, kB), kB, 0, _st, _k, h);
	YZ_LAUNCH(KCzGhostX, GridFor(_p.ny * 4, kB), kB, 0, _st, _k, h);
}

//  ConservativeUpdate (:1232-1301)
void CzStep::ConservativeUpdate(double dt)
{
	CopyGhostsH(_hNew.get());
	YZ_LAUNCH(KCzHc, GridFor(_n2, kB), kB, 0, _st, _n2, _hNew.get(), _hOld.get(), _p.theta_h, _hc.get());
	const int nf = (_p.nx - 3) * (_p.ny - 4) + (_p.nx - 4) * (_p.ny - 3);
	YZ_LAUNCH(KCzFaceFlux, GridFor(nf, kB), kB, 0, _st, _k, _hc.get(), _qCap[0].get(), _qExp[0].get(), _qCap[1].get(),
	          _qExp[1].get(), _q[0].get(), _q[1].get());
	const int nr = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KCzEnd, GridFor(nr, kB), kB, 0, _st, _k, _hOld.get(), _q[0].get(), _q[1].get(), _colSrc.get(), dt,
	          _hNew.get());
	CopyGhostsH(_hNew.get());
}

void CzStep::CalDtDh(double dt)
{
	YZ_LAUNCH(KCzDtDh, GridFor(_n2, kB), kB, 0, _st, _n2, _hNew.get(), _hOld.get(), dt, _dtdh.get());
}

void CzStep::CalVelocity(const double *fH, const double *fC)
{
	YZ_PROF("velocity", _st);
	YZ_LAUNCH(KCzVel<1>, GridFor((_p.nx - 3) * _p.ny, kB), kB, 0, _st, _k, fH, _s.get(), fC, _Ux.get());
	YZ_LAUNCH(KCzVel<0>, GridFor(_p.nx * (_p.ny - 3), kB), kB, 0, _st, _k, fH, _s.get(), fC, _Uy.get());
	YZ_LAUNCH(KCzVelGhost<1>, GridFor(_p.ny * _p.nz, kB), kB, 0, _st, _k, _Ux.get());
	YZ_LAUNCH(KCzVelGhost<0>, GridFor(_p.nx * _p.nz, kB), kB, 0, _st, _k, _Uy.get());
}

//  LocalTruncationCriterion (ImplicitSolver.cpp:271-307)
double CzStep::Lte(double dt)
{
	double th = _p.dt_criterion;
	if(std::fabs(th) <= 2.2250738585072014e-308) th = 1.0e-2;
	if(std::fabs(_dtOld) <= 2.2250738585072014e-308) return 1.0;
	const double wfloor = _p.dt_scale_floor * AbsMax(_hOld.get(), _n2);
	YZ_CUDA(cudaMemsetAsync(_max.get(), 0, sizeof(unsigned long long), _st));
	YZ_LAUNCH(KCzLte, GridFor(_n2, kB), kB, 0, _st, _n2, _hNew.get(), _hOld.get(), _hOld2.get(), _dtOld, dt, wfloor,
	          _max.get());
	unsigned long long u = 0;
	YZ_CUDA(cudaMemcpyAsync(&u, _max.get(), sizeof(u), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	double m;
	std::memcpy(&m, &u, sizeof(m));
	return 1.0 - m / th;
}

//--------------------------------------------------------------------------
//  the concentration
//--------------------------------------------------------------------------
void CzStep::BuildVolumeFluxes(const double *fH)
{
	const int nf = (_p.nx - 3) * (_p.ny - 4) + (_p.nx - 4) * (_p.ny - 3);
	YZ_LAUNCH(KCzLayerFlux, GridFor(nf, kB), kB, 0, _st, _k, fH, _Ux.get(), _Uy.get(), _q[0].get(), _q[1].get(),
	          _Qx.get(), _Qy.get());
	const int nr = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KCzZetaFlux, GridFor(nr, kB), kB, 0, _st, _k, _dtdh.get(), _Qx.get(), _Qy.get(), _colSrc.get(), _W.get());
}

void CzStep::SetBcC(const double *fH, const double *fC, bool atEnd, double dt)
{
	const int nr = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KCzBcC, GridFor(nr, kB), kB, 0, _st, _k, fH, _s.get(), fC, _W.get(), atEnd ? 1 : 0, dt, _Rc.get());
}

//  SetMatrixA (CZ_ConcEquation_2D.cpp:301-587)
void CzStep::SetMatrixAC(const double *fH, const double *fC, double dt)
{
	BuildVolumeFluxes(fH);
	const int nr = (_p.nx - 4) * (_p.ny - 4) * (_p.nz - 4);
	YZ_LAUNCH(KCzAssembleC, GridFor(nr, kB), kB, 0, _st, _k, _dRowptrC.get(), fH, _s.get(), fC, _Qx.get(), _Qy.get(),
	          _W.get(), _Ac.get(), _Bc.get(), _react.get());
	SetBcC(fH, fC, false, dt);
}

void CzStep::ApplyBoundaryRowsC(double *x)
{
	const int nr = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KCzApplyZ, GridFor(nr * 4, kB), kB, 0, _st, _k, _Rc.get(), x);
	YZ_LAUNCH(KCzApplyY, GridFor((_p.nx - 4) * 4 * _p.nz, kB), kB, 0, _st, _k, _Rc.get(), x);
	YZ_LAUNCH(KCzApplyX, GridFor(_p.ny * 4 * _p.nz, kB), kB, 0, _st, _k, _Rc.get(), x);
}

void CzStep::ExplicitPartC(const double *x, double *Ax)
{
	YZ_LAUNCH(KCzExplicit, GridFor(_n3, kB), kB, 0, _st, _n3, _dRowptrC.get(), _dColC.get(), _dBcC.get(), _Ac.get(),
	          _react.get(), x, Ax);
}

//  SolveStage (:784-892): the change d over the step, solved with the
//  solute the solve's residual leaves put back evenly over the film
int CzStep::SolveStageC(const double *fH, const double *fC, double dt, int &iter, double &resid)
{
	SetMatrixAC(fH, fC, dt);
	ApplyBoundaryRowsC(_cOld.get());
	ExplicitPartC(_cOld.get(), _Axc.get());
	const long long n3 = _n3;
	const int g = GridFor(n3, kB);
	YZ_LAUNCH(KCzMakeIA, g, kB, 0, _st, _n3, _dRowptrC.get(), _dBcC.get(), _Ac.get(), _IAc.get(), _p.theta_c, dt);
	ZeroFlag();
	YZ_LAUNCH(KCzRhsC, g, kB, 0, _st, _n3, _dBcC.get(), _Axc.get(), _Bc.get(), dt, _rhsc.get(), _flag.get());
	YZ_CUDA(cudaMemsetAsync(_d.get(), 0, (size_t)n3 * sizeof(double), _st));
	const bool any = Flag();
	int ch = 0;
	iter = 0;
	resid = 0;
	if(any)
	{
		YZ_PROF("c.linsolve", _st);
		ch = _solverC->Solve(_p.c_lin, _IAc.get(), _rhsc.get(), _d.get(), iter, resid);
		++_solves;
		_concIters += iter;
	}
	if(ch != 0)
	{
		const double m = AbsMax(_d.get(), n3);
		if(!std::isfinite(m)) YZ_CUDA(cudaMemsetAsync(_d.get(), 0, (size_t)n3 * sizeof(double), _st));
	}
	if(any && ch == 0)
	{
		//  the ghosts of d from its interior
		YZ_LAUNCH(KCzAdd, g, kB, 0, _st, n3, _cOld.get(), _d.get(), _ct.get());
		ApplyBoundaryRowsC(_ct.get());
		YZ_LAUNCH(KCzSub, g, kB, 0, _st, n3, _ct.get(), _cOld.get(), _d.get());
		YZ_LAUNCH(KCzTheta, g, kB, 0, _st, n3, _d.get(), _cOld.get(), _p.theta_c, _ct.get());
		ExplicitPartC(_ct.get(), _rhsc.get());
		YZ_LAUNCH(KCzAlpha, kRedBlocks, 256, 0, _st, _k, fH, _rhsc.get(), _Bc.get(), _d.get(), _react.get(), dt,
		          _p.theta_c, _red.get());
		YZ_LAUNCH(KCzFold2, 1, 256, 0, _st, _red.get(), _red.get() + 2 * kRedBlocks);
		double s[2];
		YZ_CUDA(cudaMemcpyAsync(s, _red.get() + 2 * kRedBlocks, sizeof(s), cudaMemcpyDeviceToHost, _st));
		YZ_CUDA(cudaStreamSynchronize(_st));
		const double alpha = (s[1] > 0.0) ? s[0] / s[1] : 0.0;
		YZ_LAUNCH(KCzShift, g, kB, 0, _st, n3, alpha, _d.get());
	}
	YZ_LAUNCH(KCzAdd, g, kB, 0, _st, n3, _cOld.get(), _d.get(), _cNew.get());
	ApplyBoundaryRowsC(_cNew.get());
	return ch;
}

//  SettleLimiter (:949-979): a limited scheme solved again at the midpoint
//  of what came out until it settles
int CzStep::SettleLimiterC(const double *fH, double dt, int &iter, double &resid)
{
	if(!_k.cI.limited) return 0;
	const long long n3 = _n3;
	const int g = GridFor(n3, kB);
	for(int pass = 0; pass < 8; ++pass)
	{
		YZ_LAUNCH(KCzMid, g, kB, 0, _st, n3, _cOld.get(), _cNew.get(), _mid.get());
		Copy(_prev.get(), _cNew.get(), (size_t)n3);
		Copy(_fC.get(), _mid.get(), (size_t)n3);
		int it = 0;
		double rs = 0;
		const int ch = SolveStageC(fH, _fC.get(), dt, it, rs);
		iter += it;
		resid = rs;
		if(ch != 0) return ch;
		YZ_CUDA(cudaMemsetAsync(_max.get(), 0, 2 * sizeof(unsigned long long), _st));
		YZ_LAUNCH(KCzLimMax, g, kB, 0, _st, n3, _cNew.get(), _prev.get(), _cOld.get(), _max.get());
		unsigned long long u[2];
		YZ_CUDA(cudaMemcpyAsync(u, _max.get(), sizeof(u), cudaMemcpyDeviceToHost, _st));
		YZ_CUDA(cudaStreamSynchronize(_st));
		double dmax, cmax;
		std::memcpy(&dmax, &u[0], sizeof(double));
		std::memcpy(&cmax, &u[1], sizeof(double));
		if(!(dmax > 1e-12 * cmax)) break;
	}
	return 0;
}

//  Solve (:911-930): a predictor, then the stage again with c halfway
int CzStep::SolveC(const double *fH, double dt, int &iter, double &resid)
{
	int ch = SolveStageC(fH, _fC.get(), dt, iter, resid);
	if(ch != 0) return ch;
	YZ_LAUNCH(KCzMid, GridFor(_n3, kB), kB, 0, _st, (long long)_n3, _cOld.get(), _cNew.get(), _fC.get());
	int it2 = 0;
	double r2 = 0;
	ch = SolveStageC(fH, _fC.get(), dt, it2, r2);
	iter += it2;
	resid = r2;
	if(ch == 0) ch = SettleLimiterC(fH, dt, iter, resid);
	Copy(_fC.get(), _cOld.get(), (size_t)_n3);
	return ch;
}

//  SolveAtMidpoint (:932-947)
int CzStep::SolveAtMidpointC(const double *fH, const double *cmid, double dt, int &iter, double &resid)
{
	Copy(_fC.get(), cmid, (size_t)_n3);
	int ch = SolveStageC(fH, _fC.get(), dt, iter, resid);
	if(ch == 0) ch = SettleLimiterC(fH, dt, iter, resid);
	Copy(_fC.get(), _cOld.get(), (size_t)_n3);
	return ch;
}

//--------------------------------------------------------------------------
//  the end of an accepted trial
//--------------------------------------------------------------------------
void CzStep::RedistributeExcess()
{
	const int nr = (_p.nx - 4) * (_p.ny - 4);
	YZ_LAUNCH(KCzExcess, GridFor(nr, kB), kB, 0, _st, _k, _cNew.get());
}

//  RedistributeDeficit (CZ_HeightEquation_2D.cpp:449-570).  The columns on
//  the device; the rare film with a column of less than no solute in all
//  takes it from the columns around on the host, as the reference does
//  (its passes are sequential over the columns)
void CzStep::RedistributeDeficit()
{
	const int nx = _p.nx, ny = _p.ny, nz = _p.nz;
	const int nr3 = (nx - 4) * (ny - 4) * (nz - 4), nr = (nx - 4) * (ny - 4);
	ZeroFlag();
	YZ_LAUNCH(KCzDeficitAny, GridFor(nr3, kB), kB, 0, _st, _k, _cNew.get(), _flag.get());
	YZ_LAUNCH(KCzDeficitCol, GridFor(nr, kB), kB, 0, _st, _k, _cNew.get(), _flag.get());
	int f[2] = {0, 0};
	YZ_CUDA(cudaMemcpyAsync(f, _flag.get(), sizeof(f), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	if(!f[0] || !f[1]) return;
	std::vector<double> c((size_t)_n3), Hv((size_t)_n2);
	_cNew.download(c.data(), c.size(), _st);
	_fH.download(Hv.data(), Hv.size(), _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
	const int kb = 2, kt = nz - 3;
	const double nLay = (double)(kt - kb + 1);
	auto I3h = [&](int i, int j, int q) { return (size_t)((q * ny + j) * nx + i); };
	auto H = [&](int i, int j) { return Hv[(size_t)(j * nx + i)]; };
	auto colMean = [&](int ix, int jy) {
		double s = 0.0;
		for(int q = kb; q <= kt; ++q) s += c[I3h(ix, jy, q)];
		return s / nLay;
	};
	auto scale = [&](int ix, int jy, double g) { for(int q = kb; q <= kt; ++q) c[I3h(ix, jy, q)] *= g; };
	auto real = [&](int ix, int jy) { return ix >= 2 && ix < nx - 2 && jy >= 2 && jy < ny - 2; };
	const int dxs[4] = {-1, 1, 0, 0}, dys[4] = {0, 0, -1, 1};
	std::vector<double> room((size_t)_n2, 0.0), take((size_t)_n2, 0.0);
	bool left = true;
	for(int pass = 0; pass < 4 && left; ++pass)
	{
		for(int ix = 2; ix < nx - 2; ++ix)
			for(int jy = 2; jy < ny - 2; ++jy)
			{
				const double m = colMean(ix, jy), h = H(ix, jy);
				room[(size_t)(jy * nx + ix)] = (m > 0.0 && h > 0.0) ? h * m : 0.0;
				take[(size_t)(jy * nx + ix)] = 0.0;
			}
		left = false;
		for(int ix = 2; ix < nx - 2; ++ix)
			for(int jy = 2; jy < ny - 2; ++jy)
			{
				const double m = colMean(ix, jy), h = H(ix, jy);
				if(!(m < 0.0)) continue;
				if(!(h > 0.0)) { scale(ix, jy, 0.0); continue; }
				const double e = -h * m;
				double r = 0.0;
				for(int q = 0; q < 4; ++q)
					if(real(ix + dxs[q], jy + dys[q])) r += room[(size_t)((jy + dys[q]) * nx + ix + dxs[q])];
				if(!(r > 0.0)) { left = true; continue; }
				const double fr = (e < r) ? e / r : 1.0;
				for(int q = 0; q < 4; ++q)
					if(real(ix + dxs[q], jy + dys[q])) take[(size_t)((jy + dys[q]) * nx + ix + dxs[q])] += fr;
				const double mNew = (fr < 1.0) ? 0.0 : -(e - r) / h;
				for(int q = kb; q <= kt; ++q) c[I3h(ix, jy, q)] = mNew;
				if(fr >= 1.0) left = true;
			}
		for(int ix = 2; ix < nx - 2; ++ix)
			for(int jy = 2; jy < ny - 2; ++jy)
			{
				const double t = take[(size_t)(jy * nx + ix)];
				if(t > 0.0)
				{
					scale(ix, jy, 1.0 - t);
					if(colMean(ix, jy) < 0.0) left = true;
				}
			}
	}
	if(left)
	{
		double lack = 0.0, total = 0.0;
		for(int ix = 2; ix < nx - 2; ++ix)
			for(int jy = 2; jy < ny - 2; ++jy)
			{
				const double m = colMean(ix, jy), h = H(ix, jy);
				if(m < 0.0) { lack -= h * m; scale(ix, jy, 0.0); }
				else if(h > 0.0) total += h * m;
			}
		const double fr = (total > 0.0) ? std::min(1.0, lack / total) : 0.0;
		if(fr > 0.0)
			for(int ix = 2; ix < nx - 2; ++ix)
				for(int jy = 2; jy < ny - 2; ++jy)
					if(H(ix, jy) > 0.0 && colMean(ix, jy) > 0.0) scale(ix, jy, 1.0 - fr);
	}
	_cNew.upload(c.data(), c.size(), _st);
}

//  AfterTimeStepTrial (CZ_HeightEquation_2D.cpp:207-386)
bool CzStep::AfterTrial(double dt, yz_cz_stats &stats)
{
	const long long n2 = _n2, n3 = _n3;
	const int g2 = GridFor(n2, kB), g3 = GridFor(n3, kB);
	ConservativeUpdate(dt);
	Copy(_fH.get(), _hNew.get(), (size_t)n2);
	_couplingPasses = 0;
	int ch = 0, iter = 0;
	double resid = 0;
	Copy(_c0.get(), _cNew.get(), (size_t)n3);
	if(_ccPrevSet)
		YZ_LAUNCH(KCzExtrap, g3, kB, 0, _st, n3, _cNew.get(), _ccPrev.get(), 0.5 * dt / _dtPrev, _cm.get());
	else
		Copy(_cm.get(), _c0.get(), (size_t)n3);
	//  what a failed step leaves as it was
	Copy(_kOld2.get(), _cOld2.get(), (size_t)n3);
	Copy(_kOld.get(), _cOld.get(), (size_t)n3);
	Copy(_kNew.get(), _cNew.get(), (size_t)n3);
	Copy(_ccPrevKeep.get(), _ccPrev.get(), (size_t)n3);
	const double dtPrevKeep = _dtPrev;
	const bool ccPrevSetKeep = _ccPrevSet;
	Copy(_ccPrev.get(), _c0.get(), (size_t)n3);
	_dtPrev = dt;
	_ccPrevSet = true;

	const int maxPass = _p.on_sc ? 1 + 8 : 1;
	double e0 = 0, e = 0, omega = 1.0;
	int pass;
	for(pass = 0; pass < maxPass; ++pass)
	{
		YZ_LAUNCH(KCzMid, g2, kB, 0, _st, n2, _hOld.get(), _hNew.get(), _hMid.get());
		if(pass > 0)
		{
			//  the film again from the start of the step, every coefficient at
			//  the midpoint the last pass found
			Copy(_fH.get(), _hMid.get(), (size_t)n2);
			Copy(_fC.get(), _cm.get(), (size_t)n3);
			int it2 = 0;
			double r2 = 0;
			SolveStageH(_fH.get(), _fC.get(), dt, it2, r2, ch);
			Copy(_fC.get(), _c0.get(), (size_t)n3);
			if(ch != 0) break;
			ConservativeUpdate(dt);
			YZ_LAUNCH(KCzMid, g2, kB, 0, _st, n2, _hOld.get(), _hNew.get(), _hMid.get());
		}
		CalDtDh(dt);
		Copy(_fH.get(), _hMid.get(), (size_t)n2);
		CalVelocity(_fH.get(), _cm.get());
		Copy(_fC.get(), _c0.get(), (size_t)n3);
		int itc = 0;
		double rc = 0;
		YZ_PROF("c.solve", _st);
		if(pass > 0) ch = SolveAtMidpointC(_fH.get(), _cm.get(), dt, itc, rc);
		else
		{
			Copy(_cOld2.get(), _cOld.get(), (size_t)n3);
			Copy(_cOld.get(), _cNew.get(), (size_t)n3);
			if(maxPass > 1) ch = SolveAtMidpointC(_fH.get(), _cm.get(), dt, itc, rc);
			else ch = SolveC(_fH.get(), dt, itc, rc) != 0 ? -1 : 0;
		}
		if(ch != 0) break;
		if(maxPass == 1) break;
		_couplingPasses = pass;
		YZ_LAUNCH(KCzCoupleRes, g3, kB, 0, _st, n3, _c0.get(), _cNew.get(), _cm.get(), _r.get());
		e = AbsMax(_r.get(), n3);
		if(pass == 0) e0 = e;
		const bool settled = !(e > 0.1 * e0) || e <= _p.coupling_floor;
		if(pass > 0 && !settled)
		{
			YZ_LAUNCH(KCzAitken, kRedBlocks, 256, 0, _st, n3, _r.get(), _rPrev.get(), _red.get());
			YZ_LAUNCH(KCzFold2, 1, 256, 0, _st, _red.get(), _red.get() + 2 * kRedBlocks);
			double s[2];
			YZ_CUDA(cudaMemcpyAsync(s, _red.get() + 2 * kRedBlocks, sizeof(s), cudaMemcpyDeviceToHost, _st));
			YZ_CUDA(cudaStreamSynchronize(_st));
			if(s[1] > 0) omega = -omega * s[0] / s[1];
		}
		if(settled) break;
		YZ_LAUNCH(KCzAxpy, g3, kB, 0, _st, n3, omega, _r.get(), _cm.get());
		Copy(_rPrev.get(), _r.get(), (size_t)n3);
	}
	if(ch == 0 && maxPass > 1 && pass == maxPass) ch = -1;
	Copy(_fH.get(), _hNew.get(), (size_t)n2);
	if(ch != 0)
	{
		Copy(_cOld2.get(), _kOld2.get(), (size_t)n3);
		Copy(_cOld.get(), _kOld.get(), (size_t)n3);
		Copy(_cNew.get(), _kNew.get(), (size_t)n3);
		Copy(_ccPrev.get(), _ccPrevKeep.get(), (size_t)n3);
		_dtPrev = dtPrevKeep;
		_ccPrevSet = ccPrevSetKeep;
		_couplingPasses = 0;
		return false;
	}
	RedistributeExcess();
	RedistributeDeficit();
	Copy(_fC.get(), _cNew.get(), (size_t)n3);
	//  RefreshGhosts: the ghosts of the end state from its own conditions
	SetBcC(_fH.get(), _fC.get(), true, dt);
	ApplyBoundaryRowsC(_cNew.get());
	Copy(_fC.get(), _cNew.get(), (size_t)n3);
	Copy(_tH.get(), _fH.get(), (size_t)n2);
	Copy(_tC.get(), _fC.get(), (size_t)n3);
	(void)stats;
	return true;
}

//--------------------------------------------------------------------------
//  TimeAdvance (CZ_HeightEquation_2D.cpp:1965-1974, SemiImplicit.cpp:100-150)
//  and the clock (TimeSteps.cpp:121-160), nsteps times
//--------------------------------------------------------------------------
void CzStep::Advance(int nsteps, yz_cz_stats &stats)
{
	YZ_CUDA(cudaSetDevice(_device));
	std::memset(&stats, 0, sizeof(stats));
	const long long l0 = t_launches, s0 = _solves, c0 = _concIters;
	const Solver::LearnedStats ls0 = _solverH->LStats();
	_lTrainMs = 0.0;
	cudaEvent_t eA, eB;
	YZ_CUDA(cudaEventCreate(&eA));
	YZ_CUDA(cudaEventCreate(&eB));
	YZ_CUDA(cudaEventRecord(eA, _st));
	const size_t n2 = (size_t)_n2, n3 = (size_t)_n3;
	for(int step = 0; step < nsteps; ++step)
	{
		YZ_PROF("step", _st);
		Copy(_hOld2.get(), _hOld.get(), n2);
		Copy(_hOld.get(), _hNew.get(), n2);
		bool done = false, failed = false;
		int iter = 0;
		double resid = 0;
		do
		{
			//  EveryTimeStepTrial: the field as the last step left it
			Copy(_fH.get(), _tH.get(), n2);
			Copy(_fC.get(), _tC.get(), n3);
			int ch = 0;
			SolveH(_dt, iter, resid, ch);
			if(_p.dt_control)
			{
				double criterion = (ch == 0) ? Lte(_dt) : -1.0;
				if(criterion > 0 && !AfterTrial(_dt, stats)) criterion = -1.0;
				//  TimeStepAdjustment (ImplicitSolver.cpp:144-190)
				double dtNext = _dt;
				if(criterion > 0.0)
				{
					done = true;
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
				done = true;
				failed = (ch != 0) || !AfterTrial(_dt, stats);
			}
		} while(!done);
		if(failed)
			throw StepFailed("ConcZ: the step did not converge at the fixed step, and with "
			                 "Numerics.TimeStepControl.Enable = false it cannot be retried at a shorter one. "
			                 "Shorten Numerics.InitialDt or enable the time-step control.");
		stats.linear_iterations += iter;
		stats.coupling_passes += _couplingPasses;
		_time += _dt;
		_dtOld = _dt;
		if(_pendingDt > 0) { _dt = _pendingDt; _pendingDt = 0; }
		stats.steps += 1;
	}
	YZ_CUDA(cudaEventRecord(eB, _st));
	YZ_CUDA(cudaEventSynchronize(eB));
	float ms = 0;
	YZ_CUDA(cudaEventElapsedTime(&ms, eA, eB));
	cudaEventDestroy(eA);
	cudaEventDestroy(eB);
	stats.time = _time;
	stats.dt = _dt;
	stats.device_ms = ms;
	stats.solves = (int)(_solves - s0);
	stats.conc_iterations = (int)(_concIters - c0);
	stats.launches = t_launches - l0;
	_launches += stats.launches;
	const Solver::LearnedStats &ls1 = _solverH->LStats();
	stats.learned_solves = ls1.solves - ls0.solves;
	stats.learned_fallbacks = ls1.fallbacks - ls0.fallbacks;
	stats.learned_iterations = ls1.iterations - ls0.iterations;
	stats.learned_samples = _learned ? _learned->Samples() : 0;
	stats.learned_train_ms = _lTrainMs;
	stats.learned_val_err = _lValErr;
	stats.learned_loss = _lLoss;
}

void CzStep::GetFields(double *h, double *c)
{
	YZ_CUDA(cudaSetDevice(_device));
	if(h) _hNew.download(h, (size_t)_n2, _st);
	if(c) _cNew.download(c, (size_t)_n3, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

//  the state a step starts from: the film and the concentration the model
//  holds (and the field and its copy at the start of the step)
void CzStep::SetFields(const double *h, const double *c)
{
	YZ_CUDA(cudaSetDevice(_device));
	if(h)
	{
		_hNew.upload(h, (size_t)_n2, _st);
		Copy(_fH.get(), _hNew.get(), (size_t)_n2);
		Copy(_tH.get(), _hNew.get(), (size_t)_n2);
	}
	if(c)
	{
		_cNew.upload(c, (size_t)_n3, _st);
		Copy(_fC.get(), _cNew.get(), (size_t)_n3);
		Copy(_tC.get(), _cNew.get(), (size_t)_n3);
	}
}

void CzStep::SetLearned(const yz_learned_cfg *cfg)
{
	YZ_CUDA(cudaSetDevice(_device));
	_solverH->SetLearned(nullptr, 0, 0, 0, 1.0);
	_learned.reset();
	_lValErr = -1.0;
	_lLoss = -1.0;
	if(!cfg) return;
	if(cfg->collect_solves < 1 || cfg->samples_per_solve < 1 || cfg->capacity < 2 || cfg->train_iters < 0 ||
	   cfg->batch < 1 || !(cfg->lr > 0) || cfg->holdout < 0 || !(cfg->cap_factor > 0) ||
	   (cfg->activation != 0 && cfg->activation != 1))
		throw UsageError("set_learned: collect_solves, samples_per_solve, batch >= 1, capacity >= 2, lr and "
		                 "cap_factor > 0, train_iters and holdout >= 0");
	_lcfg = *cfg;
	_learned.reset(new Learned(_device, _p.nx, _p.ny, cfg->capacity, cfg->seed, cfg->activation));
	_solverH->SetLearned(_learned.get(), 1, cfg->collect_solves, cfg->samples_per_solve, cfg->cap_factor);
}

//  Adam on the pairs the film's solves collected; then the film's solves try
//  the network first
void CzStep::TrainLearned()
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
	_lTrainMs += ms;
	_solverH->SetLearned(_learned.get(), 2, 0, 0, _lcfg.cap_factor);
}

void CzStep::SetPrecision(int precision)
{
	_solverH->SetPrecision(precision);
	_solverC->SetPrecision(precision);
}

void CzStep::SetTuning(int fuseFrom, int coarseLanes, int fineSweeps)
{
	_solverH->SetTuning(fuseFrom, coarseLanes, fineSweeps);
	_solverC->SetTuning(fuseFrom, coarseLanes, fineSweeps);
}

void CzStep::SetAmgReuse(int maxSolves)
{
	_solverH->SetAmgReuse(maxSolves);
	_solverC->SetAmgReuse(maxSolves);
}

//  the pieces of one step on the present state (the parity test of the
//  assemblies, the face fluxes and the velocity); the state is restored
void CzStep::Parts()
{
	YZ_CUDA(cudaSetDevice(_device));
	const size_t n2 = (size_t)_n2, n3 = (size_t)_n3;
	auto rec = [&](const char *name, const DBuf<double> &b, size_t n) {
		std::vector<double> v(n);
		b.download(v.data(), n, _st);
		YZ_CUDA(cudaStreamSynchronize(_st));
		_parts[name] = std::move(v);
	};
	DBuf<double> keepOld, keepNew;
	keepOld.reserve(n2);
	keepNew.reserve(n2);
	Copy(keepOld.get(), _hOld.get(), n2);
	Copy(keepNew.get(), _hNew.get(), n2);
	Copy(_fH.get(), _tH.get(), n2);
	Copy(_fC.get(), _tC.get(), n3);
	SetMatrixAH(_fH.get(), _fC.get(), _dt);
	rec("h_A", _A, (size_t)_nnzH);
	rec("h_B", _B, n2);
	rec("h_colsrc", _colSrc, n2);
	rec("h_qcapx", _qCap[0], n2); rec("h_qexpx", _qExp[0], n2);
	rec("h_qcapy", _qCap[1], n2); rec("h_qexpy", _qExp[1], n2);
	YZ_LAUNCH(KCzMakeIA, GridFor(_n2, kB), kB, 0, _st, _n2, _dRowptrH.get(), _dBcH.get(), _A.get(), _IA.get(),
	          _p.theta_h, _dt);
	rec("h_IA", _IA, (size_t)_nnzH);
	Copy(_hOld.get(), _hNew.get(), n2);
	ConservativeUpdate(_dt);
	rec("h_qx", _q[0], n2); rec("h_qy", _q[1], n2); rec("h_end", _hNew, n2);
	CalDtDh(_dt);
	rec("h_dtdh", _dtdh, n2);
	CalVelocity(_fH.get(), _fC.get());
	rec("ux", _Ux, n3); rec("uy", _Uy, n3);
	SetMatrixAC(_fH.get(), _fC.get(), _dt);
	rec("c_A", _Ac, (size_t)_nnzC); rec("c_B", _Bc, n3); rec("c_rhs", _Rc, n3); rec("c_react", _react, n3);
	rec("c_qx", _Qx, n3); rec("c_qy", _Qy, n3); rec("c_w", _W, n3);
	Copy(_hOld.get(), keepOld.get(), n2);
	Copy(_hNew.get(), keepNew.get(), n2);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

long long CzStep::Read(const std::string &name, double *out, long long cap)
{
	auto it = _parts.find(name);
	if(it == _parts.end()) throw UsageError("cz_read: no array '" + name + "' (yz_cz_parts first)");
	const long long n = (long long)it->second.size();
	if(out) std::memcpy(out, it->second.data(), (size_t)std::min(n, cap) * sizeof(double));
	return n;
}

int CzStep::Pattern(int which, int *rowptr, int *col, int *bc) const
{
	const std::vector<int> &rp = which ? _rowptrC : _rowptrH, &cl = which ? _colC : _colH, &b = which ? _bcC : _bcH;
	if(rowptr) std::memcpy(rowptr, rp.data(), rp.size() * sizeof(int));
	if(col) std::memcpy(col, cl.data(), cl.size() * sizeof(int));
	if(bc) std::memcpy(bc, b.data(), b.size() * sizeof(int));
	return (int)cl.size();
}

//  yz_exp_cr: the device's correctly rounded exp on host arrays
void ExpCrHost(long long n, const double *x, double *y)
{
	if(n <= 0) return;
	DBuf<double> dx, dy;
	dx.upload(x, (size_t)n, nullptr);
	dy.reserve((size_t)n);
	YZ_LAUNCH(KCrExp, GridFor(n, kB), kB, 0, nullptr, n, dx.get(), dy.get());
	dy.download(y, (size_t)n, nullptr);
	YZ_CUDA(cudaStreamSynchronize(nullptr));
}

} // namespace yz
