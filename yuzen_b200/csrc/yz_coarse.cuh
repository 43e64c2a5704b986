// yz_coarse.cuh -- the FP32 V-cycle below the finest level in one launch.
//
// The FP32 cycle's coarse part -- the restriction of the finest level's
// residual, every coarser level's pre-smoothing and residual, restriction,
// the dense solve of the coarsest level, and on the way up each level's
// prolongation and post-smoothing, ending with the prolongation to the
// finest level -- is a dozen short dependent phases per cycle, each a kernel
// of a few microseconds that the GPU mostly spends starting and draining.
// KCoarseCycle runs them all in one persistent launch: a grid that fits on
// the GPU at once (a cooperative launch), grid-stride loops over the rows of
// each phase and a grid barrier between phases.  The arithmetic of every
// phase is that of the separate kernels (yz_amg_kernels.cuh: the row sums
// with L lanes a row, the restriction with four, the dense product with a
// warp a row); the FP32 cycle's sums are not the oracle's, so the lane
// counts are the only freedom taken.
//
// The grid barrier spins with a bound: a block that waits longer than about
// a second records an error and goes on (the cycle's result is then wrong,
// and the error word tells the host).
#pragma once

#include "yz_amg_kernels.cuh"

namespace yz {

constexpr int kMaxCoarse = 12;

struct CoarseLevel
{
	int n = 0, lanes = 1, plLanes = 1, direct = 0, last = 0;
	const int *ptr = nullptr, *col = nullptr;
	const float *val = nullptr, *M = nullptr, *inv = nullptr;
	float *f = nullptr, *x = nullptr, *t = nullptr, *xt = nullptr;
	//  the restriction to the next level (its rows: the next level's n) and
	//  the prolongation from it (rows: this level's n)
	const int *rptr = nullptr, *rcol = nullptr, *pptr = nullptr, *pcol = nullptr;
	const float *rval = nullptr, *pval = nullptr;
};

struct CoarsePlan
{
	int count = 0;                 // coarse levels (1 .. count)
	//  the finest level's transfers: R0 t0 -> level 1's f, x0 + P0 x1 -> xt0
	int n0 = 0, p0Lanes = 1;
	const float *t0 = nullptr, *x0 = nullptr;
	float *xt0 = nullptr;
	const int *r0ptr = nullptr, *r0col = nullptr, *p0ptr = nullptr, *p0col = nullptr;
	const float *r0val = nullptr, *p0val = nullptr;
	CoarseLevel lv[kMaxCoarse];
};

//  bounded grid barrier (all blocks resident: a cooperative launch)
__device__ __forceinline__ void CoarseBarrier(unsigned *count, volatile unsigned *gen, int *err)
{
	__syncthreads();
	if(threadIdx.x == 0)
	{
		const unsigned g = *gen;
		__threadfence();
		if(atomicAdd(count, 1u) == gridDim.x - 1)
		{
			*count = 0u;
			__threadfence();
			atomicAdd((unsigned *)gen, 1u);
		}
		else
		{
			const long long t0 = clock64();
			while(*gen == g)
			{
				if(clock64() - t0 > 2000000000LL) { atomicExch(err, 1); break; }
			}
		}
		__threadfence();
	}
	__syncthreads();
}

//  rows of a phase, L lanes a row (32 / L rows a warp, the loop alike for a warp)
#define YZ_COARSE_ROWS(L, n)                                                                            \
	const int lane_ = threadIdx.x & 31, q = lane_ % (L);                                                \
	const long long warps_ = ((long long)gridDim.x * blockDim.x) >> 5;                                 \
	for(long long base_ = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32 / (L));      \
	    base_ < (n); base_ += warps_ * (32 / (L)))

template<int L>
__device__ void CPreRes(const CoarseLevel &c)
{
	YZ_COARSE_ROWS(L, c.n)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < c.n;
		const float s = RowSumLanes<L>(c.ptr, c.col, c.val, row, active, q, [&](int k) { return c.M[k] * c.f[k]; });
		if(active && q == 0)
		{
			const float fi = c.f[row];
			c.x[row] = c.M[row] * fi;
			c.t[row] = fi - s;
		}
	}
}

template<int L>
__device__ void CPost(const CoarseLevel &c, const float *xin, float *xout)
{
	YZ_COARSE_ROWS(L, c.n)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < c.n;
		const float s = RowSumLanes<L>(c.ptr, c.col, c.val, row, active, q, [&](int k) { return xin[k]; });
		if(active && q == 0) xout[row] = xin[row] + c.M[row] * (c.f[row] - s);
	}
}

//  y = R t (rows n), four lanes a row
__device__ void CRestrict(int n, const int *ptr, const int *col, const float *val, const float *t, float *y)
{
	YZ_COARSE_ROWS(4, n)
	{
		const long long row = base_ + lane_ / 4;
		const bool active = row < n;
		const float s = RowSumLanes<4>(ptr, col, val, row, active, q, [&](int k) { return t[k]; });
		if(active && q == 0) y[row] = s;
	}
}

//  xout = x + P xc (rows n)
template<int L>
__device__ void CProlong(int n, const int *ptr, const int *col, const float *val, const float *xc, const float *x,
                         float *xout)
{
	YZ_COARSE_ROWS(L, n)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < n;
		const float s = RowSumLanes<L>(ptr, col, val, row, active, q, [&](int k) { return xc[k]; });
		if(active && q == 0) xout[row] = x[row] + s;
	}
}
#undef YZ_COARSE_ROWS

__device__ void CDense(const CoarseLevel &c)
{
	const int lane = threadIdx.x & 31;
	const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
	for(long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c.n; i += warps)
	{
		const float *row = c.inv + (size_t)i * c.n;
		float s = 0.0f;
		for(int j = lane; j < c.n; j += 32) s = s + row[j] * c.f[j];
#pragma unroll
		for(int off = 16; off >= 1; off >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, off);
		if(lane == 0) c.x[i] = s;
	}
}

__device__ __forceinline__ void CPreResL(const CoarseLevel &c)
{
	switch(c.lanes) { case 8: CPreRes<8>(c); break; case 4: CPreRes<4>(c); break; case 2: CPreRes<2>(c); break;
	                  default: CPreRes<1>(c); break; }
}
__device__ __forceinline__ void CPostL(const CoarseLevel &c, const float *xin, float *xout)
{
	switch(c.lanes) { case 8: CPost<8>(c, xin, xout); break; case 4: CPost<4>(c, xin, xout); break;
	                  case 2: CPost<2>(c, xin, xout); break; default: CPost<1>(c, xin, xout); break; }
}
__device__ __forceinline__ void CProlongL(int lanes, int n, const int *ptr, const int *col, const float *val,
                                          const float *xc, const float *x, float *xout)
{
	switch(lanes) { case 8: CProlong<8>(n, ptr, col, val, xc, x, xout); break;
	                case 4: CProlong<4>(n, ptr, col, val, xc, x, xout); break;
	                case 2: CProlong<2>(n, ptr, col, val, xc, x, xout); break;
	                default: CProlong<1>(n, ptr, col, val, xc, x, xout); break; }
}

//  the cycle from level 1 down and back, between the finest level's
//  restriction and prolongation; bar[0] count, bar[1] generation, err
__global__ void __launch_bounds__(256) KCoarseCycle(const int *__restrict__ halt, CoarsePlan P, unsigned *bar,
                                                    int *err)
{
	if(halt && *halt) return;
	unsigned *cnt = bar;
	volatile unsigned *gen = bar + 1;
	//  down
	CRestrict(P.lv[0].n, P.r0ptr, P.r0col, P.r0val, P.t0, P.lv[0].f);
	CoarseBarrier(cnt, gen, err);
	int deepest = 0;
	for(int l = 0; l < P.count; ++l)
	{
		const CoarseLevel &c = P.lv[l];
		deepest = l;
		if(c.direct) { CDense(c); CoarseBarrier(cnt, gen, err); break; }
		if(c.last)
		{
			//  smoothed only (nothing to coarsen): x = M f, then the post-smoothing
			for(long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += (long long)gridDim.x * blockDim.x)
				c.xt[i] = c.M[i] * c.f[i];
			CoarseBarrier(cnt, gen, err);
			CPostL(c, c.xt, c.x);
			CoarseBarrier(cnt, gen, err);
			break;
		}
		CPreResL(c);
		CoarseBarrier(cnt, gen, err);
		const CoarseLevel &d = P.lv[l + 1];
		CRestrict(d.n, c.rptr, c.rcol, c.rval, c.t, d.f);
		CoarseBarrier(cnt, gen, err);
	}
	//  up
	for(int l = deepest - 1; l >= 0; --l)
	{
		const CoarseLevel &c = P.lv[l];
		CProlongL(c.plLanes, c.n, c.pptr, c.pcol, c.pval, P.lv[l + 1].x, c.x, c.xt);
		CoarseBarrier(cnt, gen, err);
		CPostL(c, c.xt, c.x);
		CoarseBarrier(cnt, gen, err);
	}
	CProlongL(P.p0Lanes, P.n0, P.p0ptr, P.p0col, P.p0val, P.lv[0].x, P.x0, P.xt0);
}

} // namespace yz
