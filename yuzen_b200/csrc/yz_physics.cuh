// yz_physics.cuh -- device restatement of the well-mixed film-height terms
// on the 2-D 13-point stencil (one thread per interior row).
//
// Stencil points are numbered as C_Grid2D::tAdjacent (model/Grids.h:161-176):
//   oM=0 mm=1 om=2 pm=3 Mo=4 mo=5 oo=6 po=7 Po=8 mp=9 op=10 pp=11 oP=12
// Directions d (GridTraits.h WM2D_Grid): 0 Xm, 1 Xp, 2 Ym, 3 Yp (axis order);
// the stencil order of directions is Ym, Xm, Xp, Yp (StencilDir).
// The sums are taken in the reference's orders (axis order, stencil order,
// stencil-point order) so that the values differ from the reference's only
// where exp / pow / log1p of the device differ from the host's in the last
// place.
#pragma once

#include <cuda_runtime.h>

namespace yz {
namespace phys {

enum { oM = 0, mm = 1, om = 2, pm = 3, Mo = 4, mo = 5, oo = 6, po = 7, Po = 8, mp = 9, op = 10, pp = 11, oP = 12 };

//  storage position of stencil point s in an interior row: A's row is the
//  capillary term's full set in FullIdx order (GridTraits.h FullIdx) with the
//  diagonal first (CRS_Matrix.h:26-29)
__host__ __device__ constexpr int Pos(int s) { return s < oo ? s + 1 : (s == oo ? 0 : s); }
__device__ __forceinline__ int AdjIdx(int d) { return d == 0 ? mo : (d == 1 ? po : (d == 2 ? om : op)); }
__device__ __forceinline__ int StencilDir(int k) { return k == 0 ? 2 : (k == 1 ? 0 : (k == 2 ? 1 : 3)); }
__device__ __forceinline__ int DirOfAdj(int idx) { return idx == mo ? 0 : (idx == po ? 1 : (idx == om ? 2 : (idx == op ? 3 : -1))); }
__device__ __forceinline__ int NarrowIdx(int k) { return k == 0 ? om : (k == 1 ? mo : (k == 2 ? oo : (k == 3 ? po : op))); }

//--------------------------------------------------------------------------
//  stencil sets of the 2-D grid (GridTraits.h WM2D_Grid)
//--------------------------------------------------------------------------
//  FaceStencil(d, q): LL, L, R, RR of face d
__host__ __device__ constexpr int FS(int d, int q)
{
	return d == 0 ? (q == 0 ? Mo : q == 1 ? mo : q == 2 ? oo : po)
	     : d == 1 ? (q == 0 ? mo : q == 1 ? oo : q == 2 ? po : Po)
	     : d == 2 ? (q == 0 ? oM : q == 1 ? om : q == 2 ? oo : op)
	              : (q == 0 ? om : q == 1 ? oo : q == 2 ? op : oP);
}
//  AxisStencil(a, q), q = 0..4
__host__ __device__ constexpr int AS(int a, int q)
{
	return a == 0 ? (q == 0 ? Mo : q == 1 ? mo : q == 2 ? oo : q == 3 ? po : Po)
	              : (q == 0 ? oM : q == 1 ? om : q == 2 ? oo : q == 3 ? op : oP);
}
//  WideIdx(k), k = 0..8
__host__ __device__ constexpr int WI(int k)
{
	return k == 0 ? oM : k == 1 ? om : k == 2 ? Mo : k == 3 ? mo : k == 4 ? oo : k == 5 ? po : k == 6 ? Po
	     : k == 7 ? op : oP;
}
__host__ __device__ constexpr bool InFace(int d, int idx)
{
	return FS(d, 0) == idx || FS(d, 1) == idx || FS(d, 2) == idx || FS(d, 3) == idx;
}
__host__ __device__ constexpr int DirOfAdjC(int idx) { return idx == mo ? 0 : idx == po ? 1 : idx == om ? 2 : idx == op ? 3 : -1; }
__host__ __device__ constexpr int StencilDirC(int k) { return k == 0 ? 2 : k == 1 ? 0 : k == 2 ? 1 : 3; }

__host__ __device__ __forceinline__ double MSign(double x) { return x >= 0 ? 1.0 : -1.0; }   // Math::Sign

//--------------------------------------------------------------------------
//  C_Interpolation_base4 (FiniteDifferences.cpp:22-213): the four-point face
//  interpolation; positions LL = 0, L = 1, R = 2, RR = 3
//--------------------------------------------------------------------------
struct Interp
{
	int kind;                 // YZ_SCHEME_*
	int limited;              // Koren or VanLeer
	double c1[4], c2[4];      // SetCoef (divided by the sum of c1)
};

//  what the assembly needs, passed by value to the kernels
struct Coef
{
	int nx, ny;
	int onL, onV, onD, onEvap;
	double theta;
	double cL[4][13];    // capillary C(d)[s]   (LaplacePressure_2D.cpp:39-94)
	double cG[4][13];    // two-point C(d)[s]   (VerticalGravityKernel.h / DisjoiningPressureKernel.h SetLinearCoef)
	double coefL, coefV, coefD;   // 1/3, -Bo/3, Dp/3
	double dx2, dy2, dx4, dy4, dx2dy2, dxx, dyy;  // FaceGradient and AddConservative spacings
	double hstar, pn, pm;
	bool slip;
	double lam, a3;             // Lambda and 3 Lambda (Mobility.h:40-46)
	double viscC0, viscBase, viscExp, sigC0, sigBase, sigCoef;
	double Ev;
	int evConc, evSpatial, evHast;
	double evMr, evMs, evPowN, evConcR, evNegExp, evNegRmax, evHast_h, evDr;
	double xmin, ymin, dx, dy, dx2h, dy2h;   // grid corner, spacing, half spacing (RectGrid.h:459-465)
	//  the upwinded terms (limited path, UpwindKernelBase.h / BodyForceKernel.h:527-691 /
	//  SolutoCapillarityKernel.h:411-516)
	int onPG, onSC, onCF;
	int wall[4];                // IsWall of the Xmin, Xmax, Ymin, Ymax edges (Symmetry, Pinning)
	int pinned[4];              // Pinning edges: no capillary flux through their wall face
	Interp hI;                  // Numerics.Convection.Height (a limited scheme)
	double pgMag[2], pgSign[2]; // Pg/3 per axis and Math::Sign(Pg)
	double cfMag, cnt[2];       // Sp/3 and the rotation axis
	double scMag;               // As*Ma/2
};

//  The face properties of a film (H, C), once per face: face f of axis a is
//  held at the index of its low cell.  vis, sig: the viscosity and surface
//  tension at the face's mean concentration; FM: Mobility::Face; DL: the
//  capillary face mobility times sig / vis; fdLH, fdHL: Face_d1 by the low /
//  the high cell; gLH, gHL: the capillary term's NonlinearJacobiProps by the
//  low / the high cell.  Every value is the one each of the two rows of the
//  face would compute (the expressions are symmetric in the two cells to
//  the bit).  piN, phN, dpN: Pi, Pi / h and dPi of every cell.
struct FaceSet
{
	double *vis, *sig, *FM, *DL, *fdLH, *fdHL, *gLH, *gHL;
};
struct FaceBuf
{
	FaceSet x, y;
	double *piN, *phN, *dpN;
};

//  what the concentration equation's kernels need (ConcEquationBase.h)
struct ConcCoef
{
	int nx, ny;
	int conv, diff;
	double th;                   // theta of the concentration equation (0.5)
	double Df, dC0, dBase, dExp; // Df and the diffusivity law
	double dxx, dyy;
	Interp cI;                   // Numerics.Convection.Concentration
};

//  WallFace (GridTraits.h:524-538) for face d of the interior cell (ix, iy)
__device__ __forceinline__ bool WallFace(const Coef &k, int d, int ix, int iy)
{
	switch(d)
	{
	case 0:  return ix == 2 && k.wall[0];
	case 1:  return ix == k.nx - 3 && k.wall[1];
	case 2:  return iy == 2 && k.wall[2];
	default: return iy == k.ny - 3 && k.wall[3];
	}
}

__device__ __forceinline__ double Limiter(int kind, double a, double b, double &pa, double &pb)
{
	double phi = 0;
	pa = 0; pb = 0;
	const bool same = (a > 0 && b > 0) || (a < 0 && b < 0);
	if(same)
	{
		if(kind == 7)
		{
			const double s = (b > 0) ? 1.0 : -1.0;
			const double aa = fabs(a), ab = fabs(b);
			const double t1 = 2.0 * aa, t2 = (2.0 * ab + aa) / 3.0, t3 = 2.0 * ab;
			if(t1 <= t2 && t1 <= t3) { phi = s * t1; pa = 2.0; pb = 0.0; }
			else if(t2 <= t3) { phi = s * t2; pa = 1.0 / 3.0; pb = 2.0 / 3.0; }
			else { phi = s * t3; pa = 0.0; pb = 2.0; }
		}
		else if(kind == 8)
		{
			const double sum = a + b;
			const double ra = a / sum, rb = b / sum;
			phi = 2.0 * a * rb;
			pa = 2.0 * rb * rb;
			pb = 2.0 * ra * ra;
		}
	}
	return phi;
}

//  The upwind side (UpwindPositions, FiniteDifferences.cpp:146-150): sign >= 0
//  takes (UU, U, D) = (LL, L, R), otherwise (RR, R, L).  Written with selects
//  so that the four values stay in registers.
__device__ __forceinline__ double FaceValue(const Interp &I, const double f[4], double sign)
{
	if(!I.limited)
	{
		double v = 0;
#pragma unroll
		for(int j = 0; j < 4; ++j) v += (I.c1[j] + MSign(sign) * I.c2[j]) * f[j];
		return v;
	}
	const bool pos = sign >= 0;
	const double fuu = pos ? f[0] : f[3], fu = pos ? f[1] : f[2], fd = pos ? f[2] : f[1];
	double pa, pb;
	return fu + 0.5 * Limiter(I.kind, fu - fuu, fd - fu, pa, pb);
}

//  rowPos: the position of the row's own cell (1 = L or 2 = R), or -1 for the
//  downwind form
__device__ __forceinline__ void FaceWeights(const Interp &I, const double f[4], double sign, int rowPos, double w[4])
{
	if(!I.limited)
	{
#pragma unroll
		for(int j = 0; j < 4; ++j) w[j] = I.c1[j] + MSign(sign) * I.c2[j];
		return;
	}
	const bool pos = sign >= 0;
	const double fuu = pos ? f[0] : f[3], fu = pos ? f[1] : f[2], fd = pos ? f[2] : f[1];
	const double a = fu - fuu, b = fd - fu;
	double pa, pb;
	const double phi = Limiter(I.kind, a, b, pa, pb);
	w[0] = 0; w[1] = 0; w[2] = 0; w[3] = 0;
	if(rowPos == (pos ? 1 : 2))
	{
		//  upwind form: f_U + chi/2 (f_U - f_UU)
		const double chi = (a != 0) ? phi / a : 0.0;
		const double wu = 1.0 + 0.5 * chi, wuu = -0.5 * chi;
		if(pos) { w[1] = wu; w[0] = wuu; }
		else { w[2] = wu; w[3] = wuu; }
	}
	else
	{
		//  downwind form: f_U + psi/2 (f_D - f_U)
		const double psi = (b != 0) ? phi / b : 0.0;
		const double wu = 1.0 - 0.5 * psi, wd = 0.5 * psi;
		if(pos) { w[1] = wu; w[2] = wd; }
		else { w[2] = wu; w[1] = wd; }
	}
}

__device__ __forceinline__ double FaceDerivative(const Interp &I, const double f[4], double sign, double g[4])
{
	if(!I.limited)
	{
#pragma unroll
		for(int j = 0; j < 4; ++j) g[j] = I.c1[j] + MSign(sign) * I.c2[j];
		return FaceValue(I, f, sign);
	}
	const bool pos = sign >= 0;
	const double fuu = pos ? f[0] : f[3], fu = pos ? f[1] : f[2], fd = pos ? f[2] : f[1];
	double pa, pb;
	const double phi = Limiter(I.kind, fu - fuu, fd - fu, pa, pb);
	const double guu = -0.5 * pa, gu = 1.0 + 0.5 * (pa - pb), gd = 0.5 * pb;
	if(pos) { g[0] = guu; g[1] = gu; g[2] = gd; g[3] = 0; }
	else { g[3] = guu; g[2] = gu; g[1] = gd; g[0] = 0; }
	return fu + 0.5 * phi;
}

//  the scheme's coefficients (FiniteDifferences.cpp:22-76)
inline Interp MakeInterp(int kind)
{
	Interp I;
	I.kind = kind;
	I.limited = (kind == 7 || kind == 8);
	double c1[4] = {0, 0, 0, 0}, c2[4] = {0, 0, 0, 0};
	switch(kind)
	{
	case 0: c1[1] = 1; c1[2] = 1; c2[1] = 1; c2[2] = -1; break;
	case 2: c1[1] = 1; c1[2] = 1; break;
	case 6: c1[0] = -1; c1[1] = 9; c1[2] = 9; c1[3] = -1; break;
	case 1: c1[0] = -1; c1[1] = 3; c1[2] = 3; c1[3] = -1; c2[0] = -1; c2[1] = 3; c2[2] = -3; c2[3] = 1; break;
	case 3: case 7: c1[0] = -1; c1[1] = 7; c1[2] = 7; c1[3] = -1; c2[0] = -1; c2[1] = 3; c2[2] = -3; c2[3] = 1; break;
	case 4: c1[0] = -1; c1[1] = 9; c1[2] = 9; c1[3] = -1; c2[0] = -1; c2[1] = 3; c2[2] = -3; c2[3] = 1; break;
	case 5: c1[0] = -1; c1[1] = 7; c1[2] = 7; c1[3] = -1; c2[0] = -1; c2[1] = 3; c2[2] = -3; c2[3] = 1; break;
	case 8: c1[0] = -1; c1[1] = 5; c1[2] = 5; c1[3] = -1; c2[0] = -1; c2[1] = 3; c2[2] = -3; c2[3] = 1; break;
	default: break;
	}
	double denom = 0;
	for(int j = 0; j < 4; ++j) denom += c1[j];
	if(kind == 5) for(int j = 0; j < 4; ++j) c2[j] *= 3.0;
	for(int j = 0; j < 4; ++j) { I.c1[j] = c1[j] / denom; I.c2[j] = c2[j] / denom; }
	return I;
}

//--------------------------------------------------------------------------
//  Mobility (model/Mobility.h)
//--------------------------------------------------------------------------
__device__ __forceinline__ double MobD(const Coef &k, double h) { const double u = fabs(h); return h * u * (u + k.a3); }
__device__ __forceinline__ double MobdD(const Coef &k, double h) { const double u = fabs(h); return u * (3.0 * u + 2.0 * k.a3); }
//  Mobility::DperH = Upwind (the slip mobility over h of an upwinded face)
__device__ __forceinline__ double MobDperH(const Coef &k, double h) { const double u = fabs(h); return u * (u + k.a3); }

__device__ inline double MobG(const Coef &k, double h)
{
	const double x = k.a3 / h;
	double f;
	if(x < 0.1)
	{
		double t = x * x, s = 0;
		for(int n = 2; n <= 18; ++n)
		{
			s += ((n % 2 == 0) ? t : -t) / n;
			t *= x;
		}
		f = s;
	}
	else f = x - log1p(x);
	return -f / (k.a3 * k.a3);
}

__device__ __forceinline__ double MobK(const Coef &k, double h)
{
	const double u = MobdD(k, h) / MobD(k, h);
	return 2.0 * u * u - (6.0 * h + 2.0 * k.a3) / MobD(k, h);
}

__device__ __forceinline__ double MobdK(const Coef &k, double h)
{
	const double d = MobD(k, h), d1 = MobdD(k, h), d2 = 6.0 * h + 2.0 * k.a3, d3 = 6.0;
	const double u = d1 / d, du = d2 / d - u * u;
	return 4.0 * u * du - (d3 * d - d2 * d1) / (d * d);
}

__device__ inline double FaceDK(const Coef &k, double h1, double h2)
{
	if(!(h1 > 0) || !(h2 > 0)) return 0;
	const double hm = 0.5 * (h1 + h2), dl = h2 - h1;
	if(fabs(dl) < 1e-3 * hm) return MobD(k, hm) / (1.0 + dl * dl * MobK(k, hm) / 24.0);
	return dl / (MobG(k, h2) - MobG(k, h1));
}

__device__ inline double FaceDK_d1(const Coef &k, double h1, double h2)
{
	if(!(h1 > 0) || !(h2 > 0)) return 0;
	const double hm = 0.5 * (h1 + h2), dl = h2 - h1;
	if(fabs(dl) < 1e-3 * hm)
	{
		const double kk = MobK(k, hm), q = 1.0 + dl * dl * kk / 24.0;
		const double Fhm = (MobdD(k, hm) * q - MobD(k, hm) * dl * dl * MobdK(k, hm) / 24.0) / (q * q);
		const double Fdl = -MobD(k, hm) * (dl * kk / 12.0) / (q * q);
		return 0.5 * Fhm - Fdl;
	}
	const double dg = MobG(k, h2) - MobG(k, h1);
	return (-dg + dl / MobD(k, h1)) / (dg * dg);
}

//  Mobility::Face / Face_d1 (positivity-preserving face mobility)
__device__ __forceinline__ double Face(const Coef &k, double h1, double h2)
{
	if(k.slip) return FaceDK(k, h1, h2);
	if(!(h1 > 0) || !(h2 > 0)) return 0;
	return 2.0 * (h1 * h1) * (h2 * h2) / (h1 + h2);
}
__device__ __forceinline__ double Face_d1(const Coef &k, double h1, double h2)
{
	if(k.slip) return FaceDK_d1(k, h1, h2);
	if(!(h1 > 0) || !(h2 > 0)) return 0;
	return 2.0 * (h1 * h2 * h2) * (h1 + h2 + h2) / ((h1 + h2) * (h1 + h2));
}

//  property laws (FluidProperty.h:100-181)
__device__ __forceinline__ double Viscosity(const Coef &k, double c) { return k.viscBase * exp(k.viscExp * (c - k.viscC0)); }
__device__ __forceinline__ double SurfaceTension(const Coef &k, double c) { return k.sigBase + k.sigCoef * (c - k.sigC0); }

//  disjoining pressure (DisjoiningPressureKernel.h:191-218)
__device__ __forceinline__ double Pi(const Coef &k, double h)
{
	if(h <= 0) return 0;
	const double r = k.hstar / h;
	return pow(r, k.pn) - pow(r, k.pm);
}
__device__ __forceinline__ double dPi(const Coef &k, double h)
{
	if(h <= 0) return 0;
	const double r = k.hstar / h;
	return -(k.pn * pow(r, k.pn) - k.pm * pow(r, k.pm)) / h;
}
__device__ __forceinline__ double PiPerH(const Coef &k, double h)
{
	if(h <= 0) return 0;
	return Pi(k, h) / h;
}

//--------------------------------------------------------------------------
//  evaporation: C_Evaporation::Evaluate (Evaporation.cpp) with Coef 1, then
//  EvapAt (HeightEquationBase.h:830-847) and SolventLimit (Evaporation.h:112)
//--------------------------------------------------------------------------
__device__ inline double NegPowFunc(const Coef &k, double rr)
{
	const double maxVal = 10, epsRmx = 1e-3;
	const double nn = k.evNegExp;
	const double kk = 0.5 * (1.0 - nn) * (2.0 - nn);
	double rev = 1.0 - rr / (k.evNegRmax * (1.0 + epsRmx));
	if(rev < 0.0 || fabs(rev) <= 2.220446049250313e-16) rev = 1e-10;   // Math::IsLessEpsilon
	const double val = kk * pow(rev, -nn);
	return val < maxVal ? val : maxVal;
}

__device__ inline double EvapRate(const Coef &k, double hh, double cc, double xx, double yy)
{
	double fMod = 1;
	if(k.evHast)
	{
		const double aa = 20.0;
		double v = (hh - k.evHast_h) / ((aa - 1.0) * k.evHast_h);
		v = v < 1.0 ? v : 1.0;
		fMod = v > 0.0 ? v : 0.0;
	}
	double fConc;
	if(k.evConc == 1)
	{
		double v = 1.0 - cc - k.evConcR;
		v = v > 0.0 ? v : 0.0;
		fConc = pow(v, k.evPowN);
	}
	else
	{
		const double c = (cc < 0.0) ? 0.0 : ((cc > 1.0) ? 1.0 : cc);
		const double chi = (c / k.evMr) / (c / k.evMr + (1.0 - c) / k.evMs);
		fConc = 1.0 - chi;
	}
	double fSp = 1.0;
	if(k.evSpatial == 1)
	{
		const double rr = sqrt(xx * xx + yy * yy);
		const double rmx = k.evNegRmax;
		const double dr = k.evDr;
		const double eps = dr * 5.0;
		const double fRE = NegPowFunc(k, rmx - eps);
		const double dU = (fRE - NegPowFunc(k, rmx - eps - dr)) / dr;
		const double aa = 2.0 * eps / 3.14159265358979323846 * dU;
		const double f0 = NegPowFunc(k, rr);
		const double rmin = rr < rmx ? rr : rmx;
		const double f1 = aa * cos(-(rmx - rmin) / eps * 0.5 * 3.14159265358979323846) + fRE;
		fSp = (rr < rmx - eps ? f0 : f1);
	}
	return 1.0 * fConc * fSp * fMod;
}

__device__ inline double EvapAt(const Coef &k, double hh, double cc, double xx, double yy, double dt)
{
	double evp = k.Ev * EvapRate(k, hh, cc, xx, yy);
	if(evp <= 0) return evp;
	if(evp * dt > 0.5 * hh) evp = (hh > 0) ? 0.5 * hh / dt : 0.0;
	if(!(evp > 0.0)) return evp;
	const double c = (cc < 0.0) ? 0.0 : ((cc > 1.0) ? 1.0 : cc);
	const double solvent = (hh > 0.0) ? hh * (1.0 - c) : 0.0;
	if(evp * dt > solvent) evp = solvent / dt;
	return evp;
}

//--------------------------------------------------------------------------
//  LaplacePressure_WM2D::FaceGradient (LaplacePressure_2D.cpp:105-128)
//--------------------------------------------------------------------------
__device__ __forceinline__ double FaceGradient(const Coef &k, const double *v, int d)
{
	const double dn4 = (d < 2) ? k.dx4 : k.dy4;
	double a1, a, b, b1, am, ap, bm, bp;
	switch(d)
	{
	case 0:  a1 = v[Mo]; a = v[mo]; b = v[oo]; b1 = v[po]; am = v[mm]; ap = v[mp]; bm = v[om]; bp = v[op]; break;
	case 1:  a1 = v[mo]; a = v[oo]; b = v[po]; b1 = v[Po]; am = v[om]; ap = v[op]; bm = v[pm]; bp = v[pp]; break;
	case 2:  a1 = v[oM]; a = v[om]; b = v[oo]; b1 = v[op]; am = v[mm]; ap = v[pm]; bm = v[mo]; bp = v[po]; break;
	default: a1 = v[om]; a = v[oo]; b = v[op]; b1 = v[oP]; am = v[mo]; ap = v[po]; bm = v[mp]; bp = v[pp]; break;
	}
	const double normal = (((b1 - b) - 2.0 * (b - a)) + (a - a1)) / dn4;
	const double cross = (((bp - b) - (b - bm)) - ((ap - a) - (a - am))) / k.dx2dy2;
	return normal + cross;
}

} // namespace phys
} // namespace yz
