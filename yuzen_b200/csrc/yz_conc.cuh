// yz_conc.cuh -- the well-mixed concentration equation on the device: the
// face volume fluxes of the film (HeightEquationBase.h:855-896), the
// concentration system of one Newton pass (ConcEquationBase.h:271-396), the
// fluxes made those of the step the film took (ConsistentFluxes,
// HeightEquationBase.h:985-1060) and the move of solute beyond [0, 1]
// (RedistributeExcess / MoveExcess, HeightEquationBase.h:1130-1275).
//
// One thread per interior row, the reference's row order and summation order
// within a row.  Sums over the whole film (the mean residual of the step, the
// solute left over after the moves) take the library's fixed reduction tree
// instead of the reference's sequential loop; they differ from it by rounding
// of the sum only.
#pragma once

#include "yz_common.cuh"
#include "yz_upwind.cuh"

namespace yz {
namespace phys {

//  Storage position of WideIdx(k) in an interior row of the concentration
//  matrix: the diagonal first, then the wide set in its order
//  (ConcEquationBase.h:243-259)
__host__ __device__ constexpr int PosC(int k) { return k < 4 ? k + 1 : (k == 4 ? 0 : k); }

__device__ __forceinline__ int OffsetOf(int s, int nx)
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

__device__ __forceinline__ double KFace(const ConcCoef &q, double ha, double hb, double ca, double cb, double dn)
{
	if(!q.diff) return 0;
	const double cm = 0.5 * (ca + cb);
	const double D = q.dBase * exp(q.dExp * (cm - q.dC0));
	return q.Df * D * (0.5 * (ha + hb)) / (dn * dn);
}

//--------------------------------------------------------------------------
//  FaceVolumeFluxes: the flux of every enabled term through the high face of
//  each interior cell (and through its low face where the cell below is a
//  ghost), summed in the order of the physics list; optionally the
//  evaporation of the step (StepSources, HeightEquationBase.h:936-965) and
//  whether the film has a cell without liquid (FilmNotPositive).
//--------------------------------------------------------------------------
__device__ __forceinline__ double FaceFluxSum(const Coef &k, const double *h, const double *c, const double *s,
                                              const double *vis, const double *DL, const double *FM, const double *pi,
                                              int d, int ix, int iy)
{
	double sum = 0;
	const int a = AdjIdx(d);
	if(k.onL) sum += k.coefL * (DL[d] * (FaceGradient(k, h, d) + FaceGradient(k, s, d)));
	if(k.onV)
	{
		const double hl = (d % 2 == 0) ? h[a] : h[oo], hh = (d % 2 == 0) ? h[oo] : h[a];
		const double sl = (d % 2 == 0) ? s[a] : s[oo], sh = (d % 2 == 0) ? s[oo] : s[a];
		const double dn = (d < 2) ? k.dxx : k.dyy;
		const double mu = vis[d];
		double gf = FM[d];
		const double tk = (gf == 0) ? 0.0 : gf / (hl + hh) / mu;
		gf /= mu;
		sum += k.coefV * ((gf * (hh - hl) + (sh - sl) * (tk * (hl + hh))) / (dn * dn));
	}
	if(k.onPG) sum += BodyForceFlux<kPG>(k, h, vis[d], d, ix, iy);
	if(k.onSC) sum += MarangoniFlux(k, h, c, vis[d], d, ix, iy);
	if(k.onCF) sum += BodyForceFlux<kCF>(k, h, vis[d], d, ix, iy);
	if(k.onD)
	{
		const double G = FM[d] / vis[d];
		const double v = k.cG[d][a] * pi[a] + k.cG[d][oo] * pi[oo];
		const double f = k.coefD * (G * v);
		sum += (d % 2 == 0) ? -f : f;
	}
	return sum;
}

__global__ void KFaceFlux(Coef k, const double *__restrict__ H, const double *__restrict__ C,
                          const double *__restrict__ S, double *__restrict__ Fx, double *__restrict__ Fy,
                          const double *__restrict__ evapOld, double dt, double *__restrict__ evp, int *filmBad,
                          FaceBuf fb)
{
	const int nx = k.nx, ny = k.ny;
	const int nIn = (nx - 4) * (ny - 4);
	int bad = 0;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nIn; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		double h[13], c[13], s[13];
#pragma unroll
		for(int q = 0; q < 13; ++q)
		{
			const int j = i + OffsetOf(q, nx);
			h[q] = H[j]; c[q] = C[j]; s[q] = S[j];
		}
		double vis[4], DL[4], FM[4], pi[13];
#pragma unroll
		for(int d = 0; d < 4; ++d)
		{
			const FaceSet f = (d < 2) ? fb.x : fb.y;
			const int fi = (d == 0) ? i - 1 : (d == 2) ? i - nx : i;
			vis[d] = f.vis[fi]; DL[d] = f.DL[fi]; FM[d] = f.FM[fi];
		}
		if(k.onD)
		{
#pragma unroll
			for(int kk = 0; kk < 5; ++kk) { const int idx = NarrowIdx(kk); pi[idx] = fb.piN[i + OffsetOf(idx, nx)]; }
		}
		//  grid y: the cell's x faces (0) or its y faces (1)
		if(blockIdx.y == 0)
		{
			Fx[i] = FaceFluxSum(k, h, c, s, vis, DL, FM, pi, 1, ix, iy);
			if(ix == 2) Fx[i - 1] = FaceFluxSum(k, h, c, s, vis, DL, FM, pi, 0, ix, iy);
		}
		else
		{
			Fy[i] = FaceFluxSum(k, h, c, s, vis, DL, FM, pi, 3, ix, iy);
			if(iy == 2) Fy[i - nx] = FaceFluxSum(k, h, c, s, vis, DL, FM, pi, 2, ix, iy);
			continue;
		}
		if(evp)
		{
			const double xx = k.xmin + ix * k.dx + k.dx2h, yy = k.ymin + iy * k.dy + k.dy2h;
			const double e = k.onEvap ? EvapAt(k, h[oo], c[oo], xx, yy, dt) : 0.0;
			evp[i] = (1.0 - k.theta) * evapOld[i] + k.theta * e;
		}
		if(!(h[oo] > 0.0)) bad = 1;
	}
	if(bad) atomicOr(filmBad, 1);
}

//--------------------------------------------------------------------------
//  The concentration system of one pass (ConcEquationBase.h:302-369): the
//  correction d = c1 - c0 of every interior row
//--------------------------------------------------------------------------
struct ConcIn
{
	const double *c0, *cLim, *h0, *h1, *cw, *F0x, *F0y, *F1x, *F1y, *evp;
	//  the nozzle's supply of the step (null: none) and whether its liquid
	//  arrives at srcConc (ConcType "supplied") or at the local c
	const double *src;
	int srcSupplied;
	double srcConc;
};

__global__ void KConcAssemble(ConcCoef q, double dt, ConcIn in, const int *__restrict__ rowptr, double *__restrict__ val,
                              double *__restrict__ rhs)
{
	const int nx = q.nx, ny = q.ny;
	const int nIn = (nx - 4) * (ny - 4);
	const double th = q.th;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nIn; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		double c0w[13], M[13];
#pragma unroll
		for(int kk = 0; kk < 9; ++kk)
		{
			const int idx = WI(kk);
			c0w[idx] = in.c0[i + OffsetOf(idx, nx)];
			M[idx] = 0;
		}
		const double c0i = c0w[oo];
		const double h1 = in.h1[i];
		//  no supply and no sideways outflow in 2-D: theta dt (r1 - S) is 0
		//  the supply (ConcEquationBase.h:310-319): at the local c, theta d
		//  of it is the new level's; at the nozzle's c, all of it is known
		const double S = in.src ? in.src[i] : 0.0;
		double diag = h1 + th * dt * (0.0 - (in.srcSupplied ? 0.0 : S));
		double R = dt * in.evp[i] * c0i;
		if(in.srcSupplied) R += dt * S * (in.srcConc - c0i);
#pragma unroll
		for(int d = 0; d < 4; ++d)
		{
			const int a = d / 2;
			const bool high = (d % 2 == 1);
			const double sg = high ? 1.0 : -1.0;
			const int adj = AdjIdx(d);
			const int ia = i + OffsetOf(adj, nx);
			const int lo = high ? i : ia;
			const double F1 = (a == 0) ? in.F1x[lo] : in.F1y[lo];
			const double F0 = (a == 0) ? in.F0x[lo] : in.F0y[lo];
			if(q.conv)
			{
				double f1[4], f0[4], w1[4], w0[4];
#pragma unroll
				for(int qq = 0; qq < 4; ++qq)
				{
					f0[qq] = c0w[FS(d, qq)];
					f1[qq] = in.cLim[i + OffsetOf(FS(d, qq), nx)];
				}
				//  the row's cell is L of its high face and R of its low one
				const int rowPos = high ? 1 : 2;
				FaceWeights(q.cI, f1, F1, rowPos, w1);
				FaceWeights(q.cI, f0, F0, rowPos, w0);
				double e1 = 0, e0 = 0;
#pragma unroll
				for(int qq = 0; qq < 4; ++qq)
				{
					M[FS(d, qq)] += th * dt * sg * F1 * w1[qq];
					e1 += w1[qq] * (f0[qq] - c0i);
					e0 += w0[qq] * (f0[qq] - c0i);
				}
				R -= dt * sg * (th * F1 * e1 + (1.0 - th) * F0 * e0);
			}
			else diag += th * dt * sg * F1;
			if(q.diff)
			{
				const double dn = (a == 0) ? q.dxx : q.dyy;
				const double K1 = KFace(q, h1, in.h1[ia], in.cw[i], in.cw[ia], dn);
				const double K0 = KFace(q, in.h0[i], in.h0[ia], c0i, c0w[adj], dn);
				diag += th * dt * K1;
				M[adj] -= th * dt * K1;
				const double dc0 = high ? (c0w[adj] - c0i) : (c0i - c0w[adj]);
				R += dt * sg * (th * K1 * dc0 + (1.0 - th) * K0 * dc0);
			}
		}
		M[oo] += diag;
		const int base = rowptr[i];
#pragma unroll
		for(int kk = 0; kk < 9; ++kk) val[base + PosC(kk)] = M[WI(kk)];
		rhs[i] = R;
	}
}

//  The boundary rows of the correction: b - L c0 with the rows [1, -1] of
//  A and their right-hand side 0 (ConcEquationBase.h:283-296)
__global__ void KConcGhostRhs(int nGhost, const int *__restrict__ ghost, const int *__restrict__ partner,
                              const double *__restrict__ c0, double *__restrict__ rhs)
{
	for(int g = blockIdx.x * blockDim.x + threadIdx.x; g < nGhost; g += gridDim.x * blockDim.x)
	{
		const int i = ghost[g], p = partner[g];
		double v = 0;
		v += 1.0 * c0[i];
		v += -1.0 * c0[p];
		rhs[i] = 0.0 - v;
	}
}

//  After a converged solve (ConcEquationBase.h:371-396 with the pass's part
//  of EveryNKLoop, HeightEquationBase.h:1428-1440): the ghosts of d by the
//  boundary rows (the next solve's guess), c1 = c0 + d with its ghosts from
//  their partners, the limiter state c1; mode 0 (a Newton pass): the working
//  field's c = min(c1, 1) and the largest move of it since the last pass;
//  mode 1 (the solves that complete the step): the largest move of c1 from
//  the limiter state it was solved with.
//  useCx: c1 and its ghosts are in cx already (the ghost rows solved
//  another way); the kernel then does the bookkeeping only
__global__ void KConcUpdate(int n, int mode, int useCx, const int *__restrict__ partnerAll, const double *__restrict__ c0,
                            double *__restrict__ d, const double *__restrict__ rhsD, double *__restrict__ cx,
                            double *__restrict__ cLim, double *__restrict__ cw, double *__restrict__ cPrev,
                            unsigned long long *maxOut)
{
	double m = 0.0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const int p = partnerAll[i];
		double x;
		if(useCx) x = cx[i];
		else if(p == i) x = c0[i] + d[i];
		else
		{
			const double dp = d[p];
			d[i] = (rhsD[i] - (-1.0 * dp)) / 1.0;
			const double xp = c0[p] + dp;
			x = (0.0 - (-1.0 * xp)) / 1.0;
		}
		cx[i] = x;
		if(mode == 0)
		{
			cLim[i] = x;
			const double cc = (x > 1.0) ? 1.0 : x;
			cw[i] = cc;
			m = fmax(m, fabs(cc - cPrev[i]));
			cPrev[i] = cc;
		}
		else
		{
			m = fmax(m, fabs(x - cLim[i]));
			cLim[i] = x;
		}
	}
	//  non-negative doubles order as their bit patterns
	unsigned long long u = (unsigned long long)__double_as_longlong(m);
	for(int off = 16; off >= 1; off >>= 1)
	{
		const unsigned long long w = __shfl_down_sync(0xffffffffu, u, off);
		u = w > u ? w : u;
	}
	if((threadIdx.x & 31) == 0 && u) atomicMax(maxOut, u);
}

//--------------------------------------------------------------------------
//  Reconstruct (ConcEquationBase.h:428-518): after a committed solve with the
//  advection, c1 of every real cell with liquid is formed once more from the
//  theta-weighted solute fluxes of its faces (SoluteFlux: the volume flux
//  times the scheme's face value of c1 and of c0, less the diffusive flux),
//  so that the sum of h c changes by the edge fluxes and the sources alone,
//  to rounding, whatever the solve's tolerance.
//--------------------------------------------------------------------------
//  the solute flux through face d of the real cell i (c1 the solve's answer
//  with its ghosts, K1 at the working field's h and c)
__device__ __forceinline__ double SoluteFluxC(const ConcCoef &q, const ConcIn &in, const double *__restrict__ c1, int i,
                                              int d)
{
	const int nx = q.nx;
	const int a = d / 2;
	const bool high = (d % 2 == 1);
	const int ia = i + OffsetOf(AdjIdx(d), nx);
	const int lo = high ? i : ia, hi = high ? ia : i;
	const double F1 = (a == 0) ? in.F1x[lo] : in.F1y[lo];
	const double F0 = (a == 0) ? in.F0x[lo] : in.F0y[lo];
	double f1[4], f0[4];
#pragma unroll
	for(int qq = 0; qq < 4; ++qq)
	{
		const int j = i + OffsetOf(FS(d, qq), nx);
		f1[qq] = c1[j];
		f0[qq] = in.c0[j];
	}
	double G1 = F1 * FaceValue(q.cI, f1, F1);
	double G0 = F0 * FaceValue(q.cI, f0, F0);
	if(q.diff)
	{
		const double dn = (a == 0) ? q.dxx : q.dyy;
		const double K1 = KFace(q, in.h1[lo], in.h1[hi], in.cw[lo], in.cw[hi], dn);
		const double K0 = KFace(q, in.h0[lo], in.h0[hi], in.c0[lo], in.c0[hi], dn);
		G1 -= K1 * (c1[hi] - c1[lo]);
		G0 -= K0 * (in.c0[hi] - in.c0[lo]);
	}
	return q.th * G1 + (1.0 - q.th) * G0;
}

//  every face once: the high faces of the real cells, and the low face of a
//  real cell whose neighbour there is a ghost (indexed by the face's low cell)
__global__ void KSoluteFaces(ConcCoef q, ConcIn in, const double *__restrict__ c1, double *__restrict__ G2x,
                             double *__restrict__ G2y)
{
	const int nx = q.nx, ny = q.ny;
	const int nIn = (nx - 4) * (ny - 4);
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nIn; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		G2x[i] = SoluteFluxC(q, in, c1, i, 1);
		G2y[i] = SoluteFluxC(q, in, c1, i, 3);
		if(ix == 2) G2x[i - 1] = SoluteFluxC(q, in, c1, i, 0);
		if(iy == 2) G2y[i - nx] = SoluteFluxC(q, in, c1, i, 2);
	}
}

//  c1 of every real cell with liquid from the faces' fluxes (c1pre: the
//  solve's answer, read; cx: written)
__global__ void KReconstruct(ConcCoef q, double dt, ConcIn in, const double *__restrict__ c1pre,
                             const double *__restrict__ G2x, const double *__restrict__ G2y, double *__restrict__ cx)
{
	const int nx = q.nx, ny = q.ny;
	const int nIn = (nx - 4) * (ny - 4);
	const double th = q.th;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < nIn; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		const double h1 = in.h1[i], h0 = in.h0[i];
		if(!(h1 > 0.0)) continue;
		double div = 0;
		div += G2x[i] - G2x[i - 1];
		div += G2y[i] - G2y[i - nx];
		const double c0 = in.c0[i];
		double qq = h0 * c0 - dt * div;
		if(in.src) qq += dt * in.src[i] * (in.srcSupplied ? in.srcConc : th * c1pre[i] + (1.0 - th) * c0);
		cx[i] = qq / h1;
	}
}

//--------------------------------------------------------------------------
//  ConsistentFluxes (HeightEquationBase.h:985-1060)
//--------------------------------------------------------------------------
//  rho of every interior cell and their sum (the library's reduction tree)
__global__ void KRho(int nx, int ny, double theta, double dt, const double *__restrict__ hOld,
                     const double *__restrict__ h1, const double *__restrict__ F1x, const double *__restrict__ F1y,
                     const double *__restrict__ F0x, const double *__restrict__ F0y, const double *__restrict__ evp,
                     const double *__restrict__ src, double *__restrict__ rho, RedScratch rs, double *sumOut)
{
	__shared__ double sh[kRT];
	const int nIn = (nx - 4) * (ny - 4);
	double a[1] = {0.0};
	const int t = blockIdx.x * kRT + threadIdx.x;
	if(t < nIn)
	{
		const int ix = 2 + t % (nx - 4), iy = 2 + t / (nx - 4);
		const int i = iy * nx + ix;
		double div1 = 0, div0 = 0;
		div1 += F1x[i] - F1x[i - 1];
		div0 += F0x[i] - F0x[i - 1];
		div1 += F1y[i] - F1y[i - nx];
		div0 += F0y[i] - F0y[i - nx];
		//  no sideways outflow in 2-D (r = 0); the nozzle's supply, if any
		const double r = (hOld[i] - h1[i]) / dt -
		                 (theta * (div1 + 0.0) + (1.0 - theta) * (div0 + 0.0) + (evp[i] - (src ? src[i] : 0.0)));
		rho[i] = r;
		a[0] = r;
	}
	double tot[1];
	if(GridFold<1>(a, sh, rs, tot) && threadIdx.x == 0) *sumOut = tot[0];
}

//  One thread per row of cells: the row's sum of rho - mean, then the x
//  faces of the row take what the y faces do not (running sums in x)
__global__ void KRowPass(int nx, int ny, double w, const double *__restrict__ rho, const double *__restrict__ sum,
                         double *__restrict__ rowSum, double *__restrict__ F1x)
{
	const int m = nx - 4;
	const int nIn = (nx - 4) * (ny - 4);
	const double mean = *sum / nIn;
	for(int jy = 2 + blockIdx.x * blockDim.x + threadIdx.x; jy <= ny - 3; jy += gridDim.x * blockDim.x)
	{
		double r = 0;
		for(int ix = 2; ix <= nx - 3; ix++) r += rho[jy * nx + ix] - mean;
		rowSum[jy] = r;
		const double share = r / m;
		double acc = 0;
		for(int ix = 2; ix < nx - 3; ix++)
		{
			acc += (rho[jy * nx + ix] - mean) - share;
			F1x[jy * nx + ix] += w * acc;
		}
	}
}

//  the running sum over the rows (one thread)
__global__ void KAccY(int nx, int ny, const double *__restrict__ rowSum, double *__restrict__ accY)
{
	if(blockIdx.x != 0 || threadIdx.x != 0) return;
	const int m = nx - 4;
	double acc = 0;
	for(int jy = 2; jy < ny - 3; jy++)
	{
		acc += rowSum[jy] / m;
		accY[jy] = acc;
	}
}

__global__ void KFyFix(int nx, int ny, double w, const double *__restrict__ accY, double *__restrict__ F1y)
{
	const int m = nx - 4, rows = ny - 5;
	for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < m * rows; t += gridDim.x * blockDim.x)
	{
		const int ix = 2 + t % m, jy = 2 + t / m;
		F1y[jy * nx + ix] += w * accY[jy];
	}
}

//--------------------------------------------------------------------------
//  RedistributeExcess / MoveExcess (HeightEquationBase.h:1130-1275).  lower:
//  below 0 (else above 1).  Every pass takes the room of every cell first,
//  moves what the cells outside the bound hold beyond it to their
//  neighbours in proportion to their room, and applies what each cell
//  receives after all have been seen: a cell's gain is summed over the
//  neighbours that give to it in the order the reference's loop visits them
//  (increasing row index).
//--------------------------------------------------------------------------
__device__ __forceinline__ bool Outside(bool lower, double c) { return lower ? (c < 0.0) : (c > 1.0); }
__device__ __forceinline__ double Beyond(bool lower, double h, double c) { return lower ? -h * c : h * (c - 1.0); }
__device__ __forceinline__ double RoomOf(bool lower, double h, double c) { return lower ? h * c : h * (1.0 - c); }

//  flags: bit 0 some interior c > 1, bit 1 some interior c < 0
__global__ void KExcessFlags(int n, const unsigned char *__restrict__ isbc, const double *__restrict__ cx, int *flags)
{
	int f = 0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(isbc[i]) continue;
		if(cx[i] > 1.0) f |= 1;
		if(cx[i] < 0.0) f |= 2;
	}
	if(f) atomicOr(flags, f);
}

__global__ void KRoom(int n, int lower, const unsigned char *__restrict__ isbc, const double *__restrict__ H,
                      const double *__restrict__ cx, double *__restrict__ room)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double h = H[i];
		const bool inside = lower ? (cx[i] > 0.0) : (cx[i] < 1.0);
		room[i] = (!isbc[i] && h > 0.0 && inside) ? RoomOf(lower, h, cx[i]) : 0.0;
	}
}

//  the cells outside: what they give (f, 0 for none), their new value;
//  flags bit 0: another pass is wanted
__global__ void KOutside(int nx, int n, int lower, int pass, const unsigned char *__restrict__ isbc,
                         const double *__restrict__ H, double *__restrict__ cx, const double *__restrict__ room,
                         double *__restrict__ give, int *flags)
{
	const double bound = lower ? 0.0 : 1.0;
	int any = 0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		give[i] = 0.0;
		if(isbc[i] || !Outside(lower, cx[i])) continue;
		const double h = H[i];
		if(!(h > 0.0)) { cx[i] = bound; continue; }
		const double e = Beyond(lower, h, cx[i]);
		double r = 0.0;
		r += room[i - 1];
		r += room[i + 1];
		r += room[i - nx];
		r += room[i + nx];
		if(!(r > 0.0)) { any = 1; continue; }
		const double f = (e < r) ? e / r : 1.0;
		give[i] = f;
		if(f < 1.0) cx[i] = bound;
		else { cx[i] = lower ? -(e - r) / h : 1.0 + (e - r) / h; any = 1; }
	}
	(void)pass;
	if(any) atomicOr(flags, 1);
}

__global__ void KGain(int nx, int n, int lower, const unsigned char *__restrict__ isbc, const double *__restrict__ H,
                      double *__restrict__ cx, const double *__restrict__ room, const double *__restrict__ give,
                      int *flags)
{
	int any = 0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(isbc[i]) continue;
		const double rm = room[i];
		double gain = 0.0;
		//  the givers in the order of their rows: below, left, right, above
		const int nb[4] = {i - nx, i - 1, i + 1, i + nx};
#pragma unroll
		for(int q = 0; q < 4; ++q)
		{
			const double f = give[nb[q]];
			if(f > 0.0) gain += f * rm;
		}
		if(gain > 0.0)
		{
			const double dc = gain / H[i];
			cx[i] += lower ? -dc : dc;
			if(Outside(lower, cx[i])) any = 1;
		}
	}
	if(any) atomicOr(flags, 1);
}

//  what is left outside after the passes and the room there is (two sums)
__global__ void KSpreadSums(int n, int lower, const unsigned char *__restrict__ isbc, const double *__restrict__ H,
                            double *__restrict__ cx, RedScratch rs, double *out)
{
	__shared__ double sh[2 * kRT];
	double a[2] = {0.0, 0.0};
	const int i = blockIdx.x * kRT + threadIdx.x;
	if(i < n && !isbc[i])
	{
		const double h = H[i];
		if(Outside(lower, cx[i])) { a[0] = Beyond(lower, h, cx[i]); cx[i] = lower ? 0.0 : 1.0; }
		else if(h > 0.0) a[1] = RoomOf(lower, h, cx[i]);
	}
	double tot[2];
	if(GridFold<2>(a, sh, rs, tot) && threadIdx.x == 0) { out[0] = tot[0]; out[1] = tot[1]; }
}

__global__ void KSpreadApply(int n, int lower, const unsigned char *__restrict__ isbc, const double *__restrict__ H,
                             double *__restrict__ cx, double f)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(isbc[i] || !(H[i] > 0.0)) continue;
		if(lower)
		{
			if(!(cx[i] > 0.0)) continue;
			cx[i] -= f * cx[i];
			if(cx[i] < 0.0) cx[i] = 0.0;
		}
		else
		{
			if(!(cx[i] < 1.0)) continue;
			cx[i] += f * (1.0 - cx[i]);
			if(cx[i] > 1.0) cx[i] = 1.0;
		}
	}
}

//  every row: above 1 set to 1; with under, below 0 set to 0
__global__ void KBoundRows(int n, int under, double *__restrict__ cx)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(cx[i] > 1.0) cx[i] = 1.0;
		if(under && cx[i] < 0.0) cx[i] = 0.0;
	}
}

//  the committed step: c0 = c1; the field's c = min(c1, 1); the limiter c1
__global__ void KConcCommit(int n, const double *__restrict__ cx, double *__restrict__ c0, double *__restrict__ cw,
                            double *__restrict__ cLim, double *__restrict__ cField)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double x = cx[i];
		c0[i] = x;
		cLim[i] = x;
		const double cc = (x > 1.0) ? 1.0 : x;
		cw[i] = cc;
		cField[i] = cc;
	}
}

} // namespace phys
} // namespace yz
