// yz_upwind.cuh -- the upwinded terms of the film-height equation, on the
// limited path (Koren, VanLeer) and on the unlimited one (the fixed
// four-point schemes, below), one interior row at a time: the in-plane gravity
// (ParallelGravityKernel.h), the rotation (CentrifugalKernel.h) and the
// Marangoni stress (SolutoCapillarityKernel.h).
//
// The flux through face j of a body force is Mag w_j h_f^3 / mu(c_f), h_f the
// limited face value of the film (C_Interpolation_base4::FaceValue).  A holds
// it as w_j (sum_q wt_q h_q) h_f^2 / mu with the weights wt frozen at the film
// (FaceWeights, downwind form), so that A(h) h is the flux to rounding; the
// Jacobian adds w_j (3 g_q - wt_q) h_f^2 / mu, g_q = dh_f/dh_q
// (BodyForceKernel.h:527-691).  The Marangoni flux Coef h_f^2 dc/mu is held
// in A as (sum_q wt_q h_q) h_f dc/mu with the Jacobian (2 g_q - wt_q) h_f dc/mu
// (SolutoCapillarityKernel.h:411-516).  Every sum is taken in the
// reference's order: axis by axis over AxisStencil for the body forces, face
// by face in axis order and then ScatterJacobiWide's order for Marangoni
// (UpwindKernelBase.h:179-213).
#pragma once

#include "yz_physics.cuh"

namespace yz {
namespace phys {

//  q of the point idx in FaceStencil(d), -1 if it is not one of them
__host__ __device__ constexpr int QOf(int d, int idx)
{
	return FS(d, 0) == idx ? 0 : FS(d, 1) == idx ? 1 : FS(d, 2) == idx ? 2 : FS(d, 3) == idx ? 3 : -1;
}

//  the body-force kinds
enum { kPG = 0, kCF = 1 };

//  FaceCoord (GridTraits.h:469-477): X / Y of face d of cell (ix, iy)
__device__ __forceinline__ double FaceCoord(const Coef &k, int d, int ix, int iy)
{
	switch(d)
	{
	case 0:  return k.xmin + ix * k.dx + 0.0;
	case 1:  return k.xmin + (ix + 1) * k.dx + 0.0;
	case 2:  return k.ymin + iy * k.dy + 0.0;
	default: return k.ymin + (iy + 1) * k.dy + 0.0;
	}
}

//  DriveFace: the direction of face d (in-plane gravity: the sign of Pg; the
//  rotation: the distance of the face from the axis)
template<int T>
__device__ __forceinline__ double DriveFace(const Coef &k, int d, int ix, int iy)
{
	if(T == kPG) return k.pgSign[d / 2];
	return FaceCoord(k, d, ix, iy) - k.cnt[d / 2];
}
//  Weight: 1 for the in-plane gravity, the distance for the rotation
template<int T>
__device__ __forceinline__ double Weight(const Coef &k, int d, int ix, int iy)
{
	if(T == kPG) return 1.0;
	return DriveFace<T>(k, d, ix, iy);
}
template<int T>
__device__ __forceinline__ double Mag(const Coef &k, int a) { return T == kPG ? k.pgMag[a] : k.cfMag; }

//  BodyForceKernel::LimitedFace: the face value hf, the weights wt / dx,
//  D = h_f^2 / mu (slip: Upwind(h_f) / mu), 0 on a wall face; with g, also
//  dh_f/dh_q / dx
//  LimitedFace on the face's own values: f its four films (LL, L, R, RR),
//  dv its drive, hs its spacing, wall whether it is a wall face
template<bool DER>
__device__ __forceinline__ void LimitedFaceF(const Coef &k, const double f[4], double vis, double dv, double hs,
                                             bool wall, double &hf, double &D, double wt[4], double g[4])
{
	if(DER)
	{
		hf = FaceDerivative(k.hI, f, dv, g);
#pragma unroll
		for(int q = 0; q < 4; ++q) g[q] /= hs;
	}
	else hf = FaceValue(k.hI, f, dv);
	FaceWeights(k.hI, f, dv, -1, wt);
#pragma unroll
	for(int q = 0; q < 4; ++q) wt[q] /= hs;
	D = (k.slip ? MobDperH(k, hf) : hf * hf) / vis;
	if(wall) D = 0;
}

template<int T, bool DER>
__device__ __forceinline__ void LimitedFace(const Coef &k, const double *h, double vis, int d, int ix, int iy,
                                            double &hf, double &D, double wt[4], double g[4])
{
	const double dv = DriveFace<T>(k, d, ix, iy);
	const double hs = (d < 2) ? k.dxx : k.dyy;
	double f[4];
#pragma unroll
	for(int q = 0; q < 4; ++q) f[q] = h[FS(d, q)];
	if(DER)
	{
		hf = FaceDerivative(k.hI, f, dv, g);
#pragma unroll
		for(int q = 0; q < 4; ++q) g[q] /= hs;
	}
	else hf = FaceValue(k.hI, f, dv);
	FaceWeights(k.hI, f, dv, -1, wt);
#pragma unroll
	for(int q = 0; q < 4; ++q) wt[q] /= hs;
	D = (k.slip ? MobDperH(k, hf) : hf * hf) / vis;
	if(WallFace(k, d, ix, iy)) D = 0;
}

//--------------------------------------------------------------------------
//  The unlimited height schemes (Upwind-1st, Central-2nd, Central-4th,
//  Upwind-2nd, UTOPIA, QUICK, Kawamura-Kuwahara; FiniteDifferences.cpp:22-76):
//  the face value is the fixed four-point combination with the upwind part
//  c2 taken by the sign of the drive, and A, the Jacobian and the flux are
//  BodyForceKernel.h:263-491 and SolutoCapillarityKernel.h:182-373.
//--------------------------------------------------------------------------

//  CellAvgCoord (GridTraits.h:488-497): the mean of the centres of the two
//  cells on either side of face d of cell (ix, iy)
__device__ __forceinline__ double CellAvgCoord(const Coef &k, int d, int ix, int iy)
{
	const double cx = k.xmin + ix * k.dx + k.dx2h, cy = k.ymin + iy * k.dy + k.dy2h;
	switch(d)
	{
	case 0:  return 0.5 * ((k.xmin + (ix - 1) * k.dx + k.dx2h) + cx);
	case 1:  return 0.5 * ((k.xmin + (ix + 1) * k.dx + k.dx2h) + cx);
	case 2:  return 0.5 * ((k.ymin + (iy - 1) * k.dy + k.dy2h) + cy);
	default: return 0.5 * ((k.ymin + (iy + 1) * k.dy + k.dy2h) + cy);
	}
}

//  Drive: the direction the face value of the unlimited path is upwinded by
//  (in-plane gravity: the sign of Pg; the rotation: the distance of the
//  cells' mean centre from the axis, CentrifugalKernel.h:87-92).  A's and
//  the Jacobian's coefficients take DriveFace's sign instead; the two agree
//  but at a face on the axis.
template<int T>
__device__ __forceinline__ double DriveCells(const Coef &k, int d, int ix, int iy)
{
	if(T == kPG) return k.pgSign[d / 2];
	return CellAvgCoord(k, d, ix, iy) - k.cnt[d / 2];
}

//  C(j) + Sign(dv) C2(j) of a body force, the coefficients divided by the
//  mesh spacing one by one (UpwindKernelBase SetUpwindCoef(true))
__device__ __forceinline__ void UnlimitedWeights(const Coef &k, double dv, double hs, double wt[4])
{
#pragma unroll
	for(int q = 0; q < 4; ++q) wt[q] = k.hI.c1[q] / hs + MSign(dv) * (k.hI.c2[q] / hs);
}

//  NonlinearTerm's face value (BodyForceKernel.h:263-302): sum_q h_q (c1 + Sign(pp) c2)
__device__ __forceinline__ double UnlimitedFaceValue(const Coef &k, const double f[4], double pp)
{
	double hh = 0;
#pragma unroll
	for(int q = 0; q < 4; ++q) hh += f[q] * (k.hI.c1[q] + MSign(pp) * k.hI.c2[q]);
	return hh;
}

//  BodyForceKernel::FaceFlux, unlimited (BodyForceKernel.h:129-147)
template<int T>
__device__ __forceinline__ double BodyForceFluxU(const Coef &k, const double *h, double vis, int d, int ix, int iy)
{
	if(WallFace(k, d, ix, iy)) return 0.0;
	const double w = Weight<T>(k, d, ix, iy);
	const double hsp = (d < 2) ? k.dxx : k.dyy;
	double f[4], wt[4];
#pragma unroll
	for(int q = 0; q < 4; ++q) f[q] = h[FS(d, q)];
	const double hh = UnlimitedFaceValue(k, f, DriveCells<T>(k, d, ix, iy));
	const double D = (k.slip ? MobDperH(k, hh) : hh * hh) / vis;
	UnlimitedWeights(k, DriveFace<T>(k, d, ix, iy), hsp, wt);
	double hs = 0;
#pragma unroll
	for(int q = 0; q < 4; ++q) hs += wt[q] * f[q];
	return Mag<T>(k, d / 2) * (w * hs * D);
}

//  BodyForceKernel::FaceFlux, limited: Mag w (sum_q wt_q h_q) D through face d
template<int T>
__device__ __forceinline__ double BodyForceFlux(const Coef &k, const double *h, double vis, int d, int ix, int iy)
{
	if(!k.hI.limited) return BodyForceFluxU<T>(k, h, vis, d, ix, iy);
	const double w = Weight<T>(k, d, ix, iy);
	double hf, D, wt[4];
	LimitedFace<T, false>(k, h, vis, d, ix, iy, hf, D, wt, nullptr);
	double hs = 0;
#pragma unroll
	for(int q = 0; q < 4; ++q) hs += wt[q] * h[FS(d, q)];
	return Mag<T>(k, d / 2) * (w * hs * D);
}

//  FaceConc (UpwindKernelBase.h:107-115): dc across face d, per spacing
__device__ __forceinline__ double FaceDc(const Coef &k, const double *c, int d)
{
	const double hsp = (d < 2) ? k.dxx : k.dyy;
	return (c[FS(d, 2)] - c[FS(d, 1)]) / hsp;
}

//  SolutoCapillarityKernel::FaceFlux, limited: Mag S (sum_q wt_q f_q) / dx
__device__ __forceinline__ double MarangoniFlux(const Coef &k, const double *h, const double *c, double vis, int d,
                                                int ix, int iy)
{
	const double dc = FaceDc(k, c, d);
	const double hsp = (d < 2) ? k.dxx : k.dyy;
	double f[4], wt[4];
#pragma unroll
	for(int q = 0; q < 4; ++q) f[q] = h[FS(d, q)];
	const double up = MSign(k.scMag) * MSign(dc);
	const double hf = FaceValue(k.hI, f, up);
	FaceWeights(k.hI, f, up, -1, wt);
	const double S = WallFace(k, d, ix, iy) ? 0.0 : (k.slip ? dc / vis * (hf + 2.0 * k.lam) : dc / vis * hf);
	double hs = 0;
#pragma unroll
	for(int q = 0; q < 4; ++q) hs += wt[q] * f[q];
	return k.scMag * (S * hs / hsp);
}

//==========================================================================
//  The limited upwind terms face by face.  Every quantity the rows take from
//  a face (its limited value, weights and derivatives, D, the drive and
//  weight, Marangoni's S and dc) depends on the face alone, and every face is
//  shared by two rows, whose A and J both need it: UpwindFaces evaluates
//  each face once (its high face for every cell that has one a row needs)
//  and stores the products the rows add, up to a sign that is the row's
//  side of the face.  The row kernels then add them in the same order as
//  BodyForceA/J and MarangoniA/J; negating a product is exact, so the sums
//  are those of the per-row evaluation (to the sign of a zero).
//
//  UpBuf: kind (0 A, 1 J) x axis x term (kPG, kCF, Marangoni) x q arrays of
//  n doubles, indexed by the face's low cell.
//==========================================================================
enum { kUpSC = 2 };
struct UpBuf
{
	double *base;
	long long stride;
	__device__ __forceinline__ double *at(int kind, int axis, int term, int q) const
	{
		return base + (long long)(((kind * 2 + axis) * 3 + term) * 4 + q) * stride;
	}
};

//  WallFace of the face whose low cell is (ix, iy) on axis a: the low wall
//  face of the first interior cell or the high one of the last
__device__ __forceinline__ bool WallFaceLow(const Coef &k, int a, int ix, int iy)
{
	if(a == 0) return (ix == 1 && k.wall[0]) || (ix == k.nx - 3 && k.wall[1]);
	return (iy == 1 && k.wall[2]) || (iy == k.ny - 3 && k.wall[3]);
}

//  one face of a body force: A's w wt_q D, J's w (r3 g_q - wt_q) D (the
//  face seen as the high face d = 2a + 1 of its low cell)
template<int T, bool J>
__device__ __forceinline__ void BodyForceFace(const Coef &k, const double f[4], double vis, int a, int ix, int iy,
                                              bool wall, const UpBuf &up, long long j)
{
	const int d = 2 * a + 1;
	const double dv = DriveFace<T>(k, d, ix, iy);
	const double hs = (d < 2) ? k.dxx : k.dyy;
	const double w = Weight<T>(k, d, ix, iy);
	const int term = (T == kPG) ? 0 : 1;
	if(!k.hI.limited)
	{
		//  SetMatrixA / SetJacobiMatrix (BodyForceKernel.h:343-491): A's
		//  w (C + Sign(dv) C2)_q D; the Jacobian adds g_q acc, g_q = dD/dh_q
		//  (NonlinearJacobi: 2 h_f c_q / mu, slip dUpwind(h_f) c_q / mu) and
		//  acc = sum_s w (C + Sign(dv) C2)_s h_s the face's A applied to h
		const double pp = DriveCells<T>(k, d, ix, iy);
		const double hh = UnlimitedFaceValue(k, f, pp);
		const double D = wall ? 0.0 : (k.slip ? MobDperH(k, hh) : hh * hh) / vis;
		double wt[4];
		UnlimitedWeights(k, dv, hs, wt);
#pragma unroll
		for(int q = 0; q < 4; ++q) up.at(0, a, term, q)[j] = w * wt[q] * D;
		if(J)
		{
			double acc = 0;
#pragma unroll
			for(int q = 0; q < 4; ++q) acc += w * wt[q] * f[q];
			const double dd = k.slip ? (hh < 0 ? -(2.0 * (-hh) + k.a3) : 2.0 * hh + k.a3) : 2.0 * hh;
#pragma unroll
			for(int q = 0; q < 4; ++q)
			{
				const double g = wall ? 0.0 : dd * (k.hI.c1[q] + MSign(pp) * k.hI.c2[q]) / vis;
				up.at(1, a, term, q)[j] = g * acc;
			}
		}
		return;
	}
	double hf, D, wt[4], g[4];
	LimitedFaceF<false>(k, f, vis, dv, hs, wall, hf, D, wt, nullptr);
#pragma unroll
	for(int q = 0; q < 4; ++q) up.at(0, a, term, q)[j] = w * wt[q] * D;
	if(J)
	{
		LimitedFaceF<true>(k, f, vis, dv, hs, wall, hf, D, wt, g);
		double r3 = 3.0;
		if(k.slip)
		{
			const double upd = MobDperH(k, hf);
			r3 = (upd != 0.0) ? MobdD(k, hf) / upd : 0.0;
		}
#pragma unroll
		for(int q = 0; q < 4; ++q) up.at(1, a, term, q)[j] = w * (r3 * g[q] - wt[q]) * D;
	}
}

//  one face of the Marangoni term: A's wt_q S / hsp, J's g_q a' with
//  a' = 1 / hsp (slip) or hf / hsp
template<bool J>
__device__ __forceinline__ void MarangoniFace(const Coef &k, const double f[4], double cl, double cr, double vis,
                                              int a, bool wall, const UpBuf &up, long long j)
{
	const double hsp = (a == 0) ? k.dxx : k.dyy;
	const double dc = (cr - cl) / hsp;
	const double upw = MSign(k.scMag) * MSign(dc);
	{
		double wt[4];
		const double hf = FaceValue(k.hI, f, upw);
		FaceWeights(k.hI, f, upw, -1, wt);
		const double S = wall ? 0.0 : (k.slip ? dc / vis * (hf + 2.0 * k.lam) : dc / vis * hf);
#pragma unroll
		for(int q = 0; q < 4; ++q) up.at(0, a, kUpSC, q)[j] = wt[q] * S / hsp;
	}
	if(J && !k.hI.limited)
	{
		//  SetJacobiMatrix, unlimited (SolutoCapillarityKernel.h:322-373):
		//  g_q a with g_q = dc / mu (C + Up C2)_q and a = sum_s (C + Up C2)_s h_s / h
		double wt[4];
		FaceWeights(k.hI, f, upw, -1, wt);
		double av = 0;
#pragma unroll
		for(int q = 0; q < 4; ++q) av += wt[q] * f[q] / hsp;
#pragma unroll
		for(int q = 0; q < 4; ++q)
		{
			const double g = wall ? 0.0 : dc / vis * wt[q];
			up.at(1, a, kUpSC, q)[j] = g * av;
		}
	}
	else if(J)
	{
		double wt[4], gd[4];
		const double hf = FaceDerivative(k.hI, f, upw, gd);
		FaceWeights(k.hI, f, upw, -1, wt);
		const double r = wall ? 0.0 : dc / vis;
		if(k.slip)
		{
			const double L2 = 2.0 * k.lam;
			const double ap = 1.0 / hsp;
#pragma unroll
			for(int q = 0; q < 4; ++q) up.at(1, a, kUpSC, q)[j] = (r * ((2.0 * hf + L2) * gd[q] - (hf + L2) * wt[q])) * ap;
		}
		else
		{
			const double ap = hf / hsp;
#pragma unroll
			for(int q = 0; q < 4; ++q) up.at(1, a, kUpSC, q)[j] = (r * (2.0 * gd[q] - wt[q])) * ap;
		}
	}
}

//  the face of direction d of row i: its low cell, axis, and the row's sign
__device__ __forceinline__ long long FaceLow(int d, long long i, int nx)
{
	return d == 0 ? i - 1 : d == 1 ? i : d == 2 ? i - nx : i;
}

//  BodyForceA from the faces: SetMatrixA_Limited (BodyForceKernel.h:595-633)
//  into the row's A_rest, axis by axis over AxisStencil
template<int T>
__device__ __forceinline__ void BodyForceAF(const Coef &k, const UpBuf &up, long long i, double *aR)
{
	const int term = (T == kPG) ? 0 : 1;
#pragma unroll
	for(int a = 0; a < 2; ++a)
	{
		const int dm = 2 * a, dp = 2 * a + 1;
		const long long jm = FaceLow(dm, i, k.nx), jp = FaceLow(dp, i, k.nx);
		const double Coef_ = Mag<T>(k, a);
#pragma unroll
		for(int q = 0; q < 5; ++q)
		{
			const int idx = AS(a, q);
			const double tm = (q < 4) ? -up.at(0, a, term, q)[jm] : 0.0;
			const double tp = (q > 0) ? up.at(0, a, term, q - 1)[jp] : 0.0;
			const double val = tm + tp;
			aR[idx] += Coef_ * val;
		}
	}
}

//  BodyForceJ from the faces: SetJacobiMatrix_Limited (BodyForceKernel.h:635-691)
template<int T>
__device__ __forceinline__ void BodyForceJF(const Coef &k, const UpBuf &up, long long i, double *J)
{
	const int term = (T == kPG) ? 0 : 1;
#pragma unroll
	for(int a = 0; a < 2; ++a)
	{
		const int dm = 2 * a, dp = 2 * a + 1;
		const long long jm = FaceLow(dm, i, k.nx), jp = FaceLow(dp, i, k.nx);
		const double Coef_ = Mag<T>(k, a);
#pragma unroll
		for(int q = 0; q < 5; ++q)
		{
			const int idx = AS(a, q);
			const double xm = (q < 4) ? -up.at(1, a, term, q)[jm] : 0.0;
			const double xp = (q > 0) ? up.at(1, a, term, q - 1)[jp] : 0.0;
			J[idx] += Coef_ * (xm + xp);
		}
	}
}

//  MarangoniA from the faces: SolutoCapillarityKernel::SetMatrixA_Limited
//  into the row's A_rest (SolutoCapillarityKernel.h:411-516)
__device__ __forceinline__ void MarangoniAF(const Coef &k, const UpBuf &up, long long i, double *aR)
{
	double Val[13];
#pragma unroll
	for(int q = 0; q < 13; ++q) Val[q] = 0;
#pragma unroll
	for(int d = 0; d < 4; ++d)
	{
		const long long jf = FaceLow(d, i, k.nx);
		const bool neg = (d % 2 == 0);
#pragma unroll
		for(int q = 0; q < 4; ++q)
		{
			const double z = up.at(0, d / 2, kUpSC, q)[jf];
			Val[FS(d, q)] += neg ? -z : z;
		}
	}
#pragma unroll
	for(int kk = 0; kk < 9; ++kk) aR[WI(kk)] += k.scMag * Val[WI(kk)];
}

//  MarangoniJ from the faces: SolutoCapillarityKernel::SetJacobiMatrix_Limited
//  with ScatterJacobiWide (UpwindKernelBase.h:179-213): the diagonal over the
//  directions in stencil order; another point: the direction that has it as
//  its neighbour first, the rest in axis order
__device__ __forceinline__ void MarangoniJF(const Coef &k, const UpBuf &up, long long i, double *J)
{
	double ga[4][4];
#pragma unroll
	for(int d = 0; d < 4; ++d)
	{
		const long long jf = FaceLow(d, i, k.nx);
		const bool neg = (d % 2 == 0);
#pragma unroll
		for(int q = 0; q < 4; ++q)
		{
			const double v = up.at(1, d / 2, kUpSC, q)[jf];
			ga[d][q] = neg ? -v : v;
		}
	}
#pragma unroll
	for(int kk = 0; kk < 9; ++kk)
	{
		const int idx = WI(kk);
		double val = 0;
		if(idx == oo)
		{
#pragma unroll
			for(int j = 0; j < 4; ++j)
			{
				const int d = StencilDirC(j);
				val += ga[d][QOf(d, oo)];
			}
		}
		else
		{
			const int first = DirOfAdjC(idx);
			if(first >= 0) val += ga[first][QOf(first, idx)];
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				if(d == first || QOf(d, idx) < 0) continue;
				val += ga[d][QOf(d, idx)];
			}
		}
		J[idx] += k.scMag * val;
	}
}

} // namespace phys
} // namespace yz
