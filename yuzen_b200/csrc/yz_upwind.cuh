// yz_upwind.cuh -- the upwinded terms of the film-height equation on the
// limited path, one interior row at a time: the in-plane gravity
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

//  SetMatrixA_Limited (BodyForceKernel.h:595-633) into the row's A_rest
template<int T>
__device__ __forceinline__ void BodyForceA(const Coef &k, const double *h, const double *vis, int ix, int iy,
                                           double *aR)
{
	double wt[4][4], D[4], w[4];
#pragma unroll
	for(int j = 0; j < 4; ++j)
	{
		double hf;
		LimitedFace<T, false>(k, h, vis[j], j, ix, iy, hf, D[j], wt[j], nullptr);
		w[j] = Weight<T>(k, j, ix, iy);
	}
#pragma unroll
	for(int a = 0; a < 2; ++a)
	{
		const int dm = 2 * a, dp = 2 * a + 1;
		const double Coef_ = Mag<T>(k, a);
#pragma unroll
		for(int q = 0; q < 5; ++q)
		{
			const int idx = AS(a, q);
			const double Wm = (q < 4) ? wt[dm][q] : 0.0;
			const double Wp = (q > 0) ? wt[dp][q - 1] : 0.0;
			const double val = -w[dm] * Wm * D[dm] + w[dp] * Wp * D[dp];
			aR[idx] += Coef_ * val;
		}
	}
}

//  SetJacobiMatrix_Limited (BodyForceKernel.h:635-691)
template<int T>
__device__ __forceinline__ void BodyForceJ(const Coef &k, const double *h, const double *vis, int ix, int iy,
                                           double *J)
{
	double X[4][4];
#pragma unroll
	for(int j = 0; j < 4; ++j)
	{
		double hf, D, wt[4], g[4];
		LimitedFace<T, true>(k, h, vis[j], j, ix, iy, hf, D, wt, g);
		double r3 = 3.0;
		if(k.slip)
		{
			const double up = MobDperH(k, hf);
			r3 = (up != 0.0) ? MobdD(k, hf) / up : 0.0;
		}
		const double sg = (j % 2 == 0) ? -1.0 : +1.0;
		const double w = Weight<T>(k, j, ix, iy);
#pragma unroll
		for(int q = 0; q < 4; ++q) X[j][q] = sg * w * (r3 * g[q] - wt[q]) * D;
	}
#pragma unroll
	for(int a = 0; a < 2; ++a)
	{
		const int dm = 2 * a, dp = 2 * a + 1;
		const double Coef_ = Mag<T>(k, a);
#pragma unroll
		for(int q = 0; q < 5; ++q)
		{
			const int idx = AS(a, q);
			const double xm = (q < 4) ? X[dm][q] : 0.0;
			const double xp = (q > 0) ? X[dp][q - 1] : 0.0;
			J[idx] += Coef_ * (xm + xp);
		}
	}
}

//  BodyForceKernel::FaceFlux, limited: Mag w (sum_q wt_q h_q) D through face d
template<int T>
__device__ __forceinline__ double BodyForceFlux(const Coef &k, const double *h, double vis, int d, int ix, int iy)
{
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

//  SolutoCapillarityKernel::SetMatrixA_Limited into the row's A_rest
__device__ __forceinline__ void MarangoniA(const Coef &k, const double *h, const double *c, const double *vis, int ix,
                                           int iy, double *aR)
{
	double Val[13];
#pragma unroll
	for(int q = 0; q < 13; ++q) Val[q] = 0;
#pragma unroll
	for(int d = 0; d < 4; ++d)
	{
		const double dc = FaceDc(k, c, d);
		double f[4], wt[4];
#pragma unroll
		for(int q = 0; q < 4; ++q) f[q] = h[FS(d, q)];
		const double up = MSign(k.scMag) * MSign(dc);
		const double hf = FaceValue(k.hI, f, up);
		FaceWeights(k.hI, f, up, -1, wt);
		const double S = WallFace(k, d, ix, iy) ? 0.0 : (k.slip ? dc / vis[d] * (hf + 2.0 * k.lam) : dc / vis[d] * hf);
		const double hsp = (d < 2) ? k.dxx : k.dyy;
		const double sg = (d % 2 == 0) ? -1.0 : +1.0;
#pragma unroll
		for(int q = 0; q < 4; ++q) Val[FS(d, q)] += sg * wt[q] * S / hsp;
	}
#pragma unroll
	for(int kk = 0; kk < 9; ++kk) aR[WI(kk)] += k.scMag * Val[WI(kk)];
}

//  SolutoCapillarityKernel::SetJacobiMatrix_Limited with ScatterJacobiWide
__device__ __forceinline__ void MarangoniJ(const Coef &k, const double *h, const double *c, const double *vis, int ix,
                                           int iy, double *J)
{
	double a[4], g[4][4];
#pragma unroll
	for(int d = 0; d < 4; ++d)
	{
		const double dc = FaceDc(k, c, d);
		double f[4], wt[4], gd[4];
#pragma unroll
		for(int q = 0; q < 4; ++q) f[q] = h[FS(d, q)];
		const double up = MSign(k.scMag) * MSign(dc);
		const double hf = FaceDerivative(k.hI, f, up, gd);
		FaceWeights(k.hI, f, up, -1, wt);
		const double r = WallFace(k, d, ix, iy) ? 0.0 : dc / vis[d];
		const double hsp = (d < 2) ? k.dxx : k.dyy;
		const double sg = (d % 2 == 0) ? -1.0 : +1.0;
		if(k.slip)
		{
			const double L2 = 2.0 * k.lam;
			a[d] = sg / hsp;
#pragma unroll
			for(int q = 0; q < 4; ++q) g[d][q] = r * ((2.0 * hf + L2) * gd[q] - (hf + L2) * wt[q]);
		}
		else
		{
			a[d] = sg * hf / hsp;
#pragma unroll
			for(int q = 0; q < 4; ++q) g[d][q] = r * (2.0 * gd[q] - wt[q]);
		}
	}
	//  ScatterJacobiWide: the diagonal over the directions in stencil order;
	//  another point: the direction that has it as its neighbour first, the
	//  rest in axis order
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
				val += g[d][QOf(d, oo)] * a[d];
			}
		}
		else
		{
			const int first = DirOfAdjC(idx);
			if(first >= 0) val += g[first][QOf(first, idx)] * a[first];
#pragma unroll
			for(int d = 0; d < 4; ++d)
			{
				if(d == first || QOf(d, idx) < 0) continue;
				val += g[d][QOf(d, idx)] * a[d];
			}
		}
		J[idx] += k.scMag * val;
	}
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

} // namespace phys
} // namespace yz
