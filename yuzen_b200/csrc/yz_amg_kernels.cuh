// yz_amg_kernels.cuh -- device kernels of the smoothed-aggregation AMG set-up
// and V-cycle.  Every floating-point expression follows the oracle
// (oracle/solver/yzo_solver.cpp) operation for operation; the file is compiled
// with -fmad=false so that no product is fused into an addition.
#pragma once

#include "yz_common.cuh"

namespace yz {

enum : int { kOut = 0, kUndecided = 1, kIn = 2 };

__device__ __forceinline__ uint32_t Hash32(uint32_t x)
{
	x ^= x >> 16; x *= 0x85ebca6bu;
	x ^= x >> 13; x *= 0xc2b2ae35u;
	x ^= x >> 16;
	return x;
}

__device__ __forceinline__ unsigned long long PackKey(int state, int i)
{
	return ((unsigned long long)state << 62) |
	       ((unsigned long long)(Hash32((uint32_t)i) & 0x3fffffffu) << 32) |
	       (unsigned long long)(uint32_t)i;
}

//--------------------------------------------------------------------------
//  Row access of the finest level.  Its matrix is held twice: CSR for the
//  set-up, and sliced ELLPACK (slices of 32 rows, entry k of every row of a
//  slice side by side, SELL-32) for the kernels of the iterations, whose
//  loads a warp then makes as whole lines.  A row's entries are taken in
//  the same order either way (ascending column), so every sum is the same.
//  sellOff null: CSR.
//--------------------------------------------------------------------------
__device__ __forceinline__ void RowRange(const int *__restrict__ ptr, const int *__restrict__ sellOff, int i, int &start,
                                         int &len, int &stride)
{
	len = ptr[i + 1] - ptr[i];
	if(sellOff) { start = sellOff[i >> 5] + (i & 31); stride = 32; }
	else { start = ptr[i]; stride = 1; }
}

//  sum_k val[e_k] * X(col[e_k]) over a row (e_k = st + k stride), from 0 in
//  the row's order: the loads of four entries are issued together and the
//  products then added one after the other, so the sum is the sequential
//  one with four loads in flight instead of one.  T is the arithmetic (the
//  type of the values): double everywhere but in the FP32 V-cycle.
//  The values may be stored narrower than the arithmetic (float values in a
//  double sum: the FP32-matrix SpMV); the arithmetic is that of X.
template<class V, class XF>
__device__ __forceinline__ auto RowSum(int st, int len, int sd, const int *__restrict__ col, const V *__restrict__ val,
                                       XF xf) -> decltype(xf(0))
{
	using T = decltype(xf(0));
	T s = T(0);
	int k = 0, e = st;
	for(; k + 4 <= len; k += 4, e += 4 * sd)
	{
		const int c0 = col[e], c1 = col[e + sd], c2 = col[e + 2 * sd], c3 = col[e + 3 * sd];
		const T v0 = (T)val[e], v1 = (T)val[e + sd], v2 = (T)val[e + 2 * sd], v3 = (T)val[e + 3 * sd];
		const T x0 = xf(c0), x1 = xf(c1), x2 = xf(c2), x3 = xf(c3);
		s = s + v0 * x0;
		s = s + v1 * x1;
		s = s + v2 * x2;
		s = s + v3 * x3;
	}
	for(; k < len; ++k, e += sd) s = s + (T)val[e] * xf(col[e]);
	return s;
}

//  RowSum of row i of the finest level (SELL-32, entry k at st + 32 k).  A
//  stencil row's loop is unrolled to the 16 entries a stencil may have, so
//  that every offset is read from the kernel's parameters by a constant
//  index; the sum is the same sequential one.
template<class V, class XF>
__device__ __forceinline__ auto RowSumSten(const Sten &sn, int i, int st, int len, int sd, const int *__restrict__ col,
                                           const V *__restrict__ val, XF xf) -> decltype(xf(0))
{
	using T = decltype(xf(0));
	if(sn.slice && sn.slice[i >> 5])
	{
		T s = T(0);
#pragma unroll
		for(int k0 = 0; k0 < 16; k0 += 4)
		{
			if(k0 >= len) break;
			T v[4], xv[4];
#pragma unroll
			for(int j = 0; j < 4; ++j)
				if(k0 + j < len) { v[j] = (T)val[st + (k0 + j) * sd]; xv[j] = xf(i + sn.off[k0 + j]); }
#pragma unroll
			for(int j = 0; j < 4; ++j)
				if(k0 + j < len) s = s + v[j] * xv[j];
		}
		return s;
	}
	return RowSum(st, len, sd, col, val, xf);
}

//--------------------------------------------------------------------------
//  ScaleRows + gather into the sorted mirror (LinearSolverBackend.cpp:227-252),
//  into both layouts of the finest level
//--------------------------------------------------------------------------
__global__ void KScaleGather(int n, const int *__restrict__ rowptr, const int *__restrict__ ssrc,
                             const double *__restrict__ values, const double *__restrict__ rhs, int scaling,
                             double *__restrict__ val0, double *__restrict__ b, const int *__restrict__ sellOff,
                             double *__restrict__ sellVal, float *__restrict__ sellVal32)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const int st = rowptr[i], ed = rowptr[i + 1];
		const int so = sellOff[i >> 5] + (i & 31);
		const double d = scaling ? values[st] : 1.0;
		if(!scaling || fabs(d) < 1.0e-30)
		{
			for(int k = st; k < ed; ++k)
			{
				const double v = values[ssrc[k]];
				val0[k] = v;
				sellVal[so + 32 * (k - st)] = v;
				if(sellVal32) sellVal32[so + 32 * (k - st)] = (float)v;
			}
			b[i] = rhs[i];
			continue;
		}
		const double inv = 1.0 / d;
		for(int k = st; k < ed; ++k)
		{
			const double v = values[ssrc[k]] * inv;
			val0[k] = v;
			sellVal[so + 32 * (k - st)] = v;
			if(sellVal32) sellVal32[so + 32 * (k - st)] = (float)v;
		}
		b[i] = rhs[i] * inv;
	}
}

//--------------------------------------------------------------------------
//  strength of connection, aggregation
//--------------------------------------------------------------------------
__global__ void KDiag(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                      const double *__restrict__ val, double *__restrict__ dia)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		double d = 0.0;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k) if(col[k] == i) { d = val[k]; break; }
		dia[i] = d;
	}
}

__global__ void KStrength(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                          const double *__restrict__ val, const double *__restrict__ dia, double eps2,
                          unsigned char *__restrict__ strong, int *__restrict__ icnt)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double e = eps2 * dia[i];
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
		{
			const int c = col[k];
			const double v = val[k];
			const bool s = (c != i) && (e * dia[c] < v * v);
			strong[k] = s ? 1 : 0;
			if(s) atomicAdd(&icnt[c], 1);
		}
	}
}

//  in-neighbours (rows that hold this one strongly); the order inside a list
//  is free, every later use is a max or a min over it
__global__ void KFillIn(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                        const unsigned char *__restrict__ strong, int *__restrict__ ifill, int *__restrict__ icol)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
			if(strong[k]) icol[atomicAdd(&ifill[col[k]], 1)] = i;
}

__global__ void KMisInit(int n, const int *__restrict__ ptr, const unsigned char *__restrict__ strong,
                         const int *__restrict__ iptr, int *__restrict__ state, unsigned char *__restrict__ iso)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		bool any = iptr[i + 1] > iptr[i];
		for(int k = ptr[i]; k < ptr[i + 1] && !any; ++k) any = strong[k] != 0;
		iso[i] = any ? 0 : 1;
		state[i] = any ? kUndecided : kOut;
	}
}

//  The rounds of the distance-2 independent set.  Round r reads the count of
//  undecided rows u[r & 1] (0: the set is complete, the round does nothing),
//  takes the largest key within distance 2 (KMisMax twice), and KMisUpdate
//  decides the rows, writes the keys of the next round over the maxima it
//  has read and counts the rows still undecided into u[(r + 1) & 1], which
//  the round's first KMisMax has zeroed.
__global__ void KMisPack(int n, const int *__restrict__ state, unsigned long long *__restrict__ T0, int *__restrict__ undecided)
{
	int cnt = 0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		T0[i] = PackKey(state[i], i);
		cnt += (state[i] == kUndecided);
	}
	for(int off = 16; off >= 1; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
	if((threadIdx.x & 31) == 0 && cnt) atomicAdd(undecided, cnt);
}

__global__ void KMisMax(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                        const unsigned char *__restrict__ strong, const int *__restrict__ iptr,
                        const int *__restrict__ icol, const unsigned long long *__restrict__ Tin,
                        unsigned long long *__restrict__ Tout, const int *__restrict__ undecided, int *zero)
{
	if(zero && blockIdx.x == 0 && threadIdx.x == 0) *zero = 0;
	if(*undecided == 0) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		unsigned long long m = Tin[i];
		for(int k = ptr[i]; k < ptr[i + 1]; ++k) if(strong[k]) { const unsigned long long u = Tin[col[k]]; m = u > m ? u : m; }
		for(int k = iptr[i]; k < iptr[i + 1]; ++k) { const unsigned long long u = Tin[icol[k]]; m = u > m ? u : m; }
		Tout[i] = m;
	}
}

__global__ void KMisUpdate(int n, int *__restrict__ state, unsigned long long *__restrict__ T2, const int *__restrict__ undecided,
                           int *__restrict__ nextUndecided)
{
	if(*undecided == 0) return;
	int cnt = 0;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		int st = state[i];
		if(st == kUndecided)
		{
			const unsigned long long t = T2[i];
			if((int)(uint32_t)(t & 0xffffffffull) == i) st = kIn;
			else if((int)(t >> 62) == kIn) st = kOut;
			state[i] = st;
		}
		T2[i] = PackKey(st, i);
		cnt += (st == kUndecided);
	}
	for(int off = 16; off >= 1; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
	if((threadIdx.x & 31) == 0 && cnt) atomicAdd(nextUndecided, cnt);
}

__global__ void KRootFlags(int n, const int *__restrict__ state, int *__restrict__ flag)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = state[i] == kIn ? 1 : 0;
}

__global__ void KAssignFirst(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                             const unsigned char *__restrict__ strong, const int *__restrict__ iptr,
                             const int *__restrict__ icol, const int *__restrict__ state,
                             const unsigned char *__restrict__ iso, const int *__restrict__ rootId, int *__restrict__ first)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(state[i] == kIn) { first[i] = rootId[i]; continue; }
		if(iso[i]) { first[i] = -1; continue; }
		int best = -1;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
			if(strong[k]) { const int j = col[k]; if(state[j] == kIn && (best < 0 || rootId[j] < best)) best = rootId[j]; }
		for(int k = iptr[i]; k < iptr[i + 1]; ++k)
		{ const int j = icol[k]; if(state[j] == kIn && (best < 0 || rootId[j] < best)) best = rootId[j]; }
		first[i] = best;
	}
}

__global__ void KAssignSecond(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                              const unsigned char *__restrict__ strong, const int *__restrict__ iptr,
                              const int *__restrict__ icol, const unsigned char *__restrict__ iso,
                              const int *__restrict__ first, int *__restrict__ agg)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(first[i] >= 0 || iso[i]) { agg[i] = first[i]; continue; }
		int best = -1;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
			if(strong[k]) { const int f = first[col[k]]; if(f >= 0 && (best < 0 || f < best)) best = f; }
		for(int k = iptr[i]; k < iptr[i + 1]; ++k)
		{ const int f = first[icol[k]]; if(f >= 0 && (best < 0 || f < best)) best = f; }
		agg[i] = best;
	}
}

__global__ void KSpai0(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                       const double *__restrict__ val, double *__restrict__ M)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		double num = 0.0, den = 0.0;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
		{
			const double v = val[k];
			den = den + v * v;
			if(col[k] == i) num = num + v;
		}
		M[i] = (1.0 / den) * num;
	}
}

//  damped Jacobi as a preconditioner: m_i = 0.72 * (1 / a_ii)
__global__ void KDampedJacobi(int n, const double *__restrict__ dia, double *__restrict__ M)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) M[i] = 0.72 * (1.0 / dia[i]);
}

//--------------------------------------------------------------------------
//  prolongation  P = (I - omega D_f^-1 A_f) P_tent
//--------------------------------------------------------------------------
constexpr int kRowCap = 256;	// distinct aggregates / columns a row may gather

//  CAP: the distinct aggregates a row may gather in this launch (a row of A
//  with more entries than CAP sets *overflow; the caller then launches the
//  kRowCap instance)
template<int CAP>
__global__ void KPCount(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                        const unsigned char *__restrict__ strong, const int *__restrict__ agg,
                        int *__restrict__ cnt, int *__restrict__ overflow)
{
	int lc[CAP];
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		int m = 0;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
		{
			const int c = col[k];
			if(c != i && !strong[k]) continue;
			const int cp = agg[c];
			if(cp < 0) continue;
			int q = 0;
			while(q < m && lc[q] != cp) ++q;
			if(q == m) { if(m == CAP) { atomicExch(overflow, 1); break; } lc[m++] = cp; }
		}
		cnt[i] = m;
	}
}

template<int CAP>
__global__ void KPFill(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                       const double *__restrict__ val, const unsigned char *__restrict__ strong,
                       const int *__restrict__ agg, const int *__restrict__ pptr,
                       int *__restrict__ pcol, double *__restrict__ pval)
{
	const double omega = 2.0 / 3.0;
	int lc[CAP];
	double lv[CAP];
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		double dia = 0.0;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
			if(col[k] == i || !strong[k]) dia = dia + val[k];
		const double ds = (-omega) * (1.0 / dia);
		int m = 0;
		for(int k = ptr[i]; k < ptr[i + 1]; ++k)
		{
			const int c = col[k];
			if(c != i && !strong[k]) continue;
			const int cp = agg[c];
			if(cp < 0) continue;
			const double va = (c == i) ? (1.0 - omega) : ds * val[k];
			int q = 0;
			while(q < m && lc[q] != cp) ++q;
			if(q == m) { if(m == CAP) break; lc[m] = cp; lv[m] = 0.0; ++m; }
			lv[q] = lv[q] + va;
		}
		//  insertion sort by column (columns are distinct)
		for(int a = 1; a < m; ++a)
		{
			const int kc = lc[a]; const double kv = lv[a];
			int b = a - 1;
			while(b >= 0 && lc[b] > kc) { lc[b + 1] = lc[b]; lv[b + 1] = lv[b]; --b; }
			lc[b + 1] = kc; lv[b + 1] = kv;
		}
		const int o = pptr[i];
		for(int q = 0; q < m; ++q) { pcol[o + q] = lc[q]; pval[o + q] = lv[q]; }
	}
}

//  R = P^T: counts per column, atomic fill, then each row sorted by fine row
__global__ void KColCount(int nnz, const int *__restrict__ pcol, int *__restrict__ cnt)
{
	for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) atomicAdd(&cnt[pcol[k]], 1);
}

__global__ void KTransposeFill(int n, const int *__restrict__ pptr, const int *__restrict__ pcol,
                               const double *__restrict__ pval, int *__restrict__ fill,
                               int *__restrict__ rcol, double *__restrict__ rval)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		for(int k = pptr[i]; k < pptr[i + 1]; ++k)
		{
			const int d = atomicAdd(&fill[pcol[k]], 1);
			rcol[d] = i; rval[d] = pval[k];
		}
}

//  each row sorted by column (the columns of a row are distinct): one warp
//  per row, every entry placed at its rank among the row's columns (rows of
//  up to 64 entries), longer rows by insertion in place
__global__ void __launch_bounds__(256) KRowSort(int n, const int *__restrict__ ptr, int *__restrict__ col,
                                                double *__restrict__ val)
{
	constexpr int L = 64, W = 8;
	__shared__ int sc[W][L];
	__shared__ double sv[W][L];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
	for(long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps)
	{
		const int i = (int)row;
		const int st = ptr[i], ed = ptr[i + 1], m = ed - st;
		if(m <= L)
		{
			for(int a2 = lane; a2 < m; a2 += 32) { sc[w][a2] = col[st + a2]; sv[w][a2] = val[st + a2]; }
			__syncwarp();
			for(int a2 = lane; a2 < m; a2 += 32)
			{
				const int cc = sc[w][a2];
				int r = 0;
				for(int b2 = 0; b2 < m; ++b2) r += (sc[w][b2] < cc);
				col[st + r] = cc; val[st + r] = sv[w][a2];
			}
			__syncwarp();
			continue;
		}
		if(lane != 0) continue;
		for(int a2 = st + 1; a2 < ed; ++a2)
		{
			const int kc = col[a2]; const double kv = val[a2];
			int b2 = a2 - 1;
			while(b2 >= st && col[b2] > kc) { col[b2 + 1] = col[b2]; val[b2 + 1] = val[b2]; --b2; }
			col[b2 + 1] = kc; val[b2 + 1] = kv;
		}
	}
}

//--------------------------------------------------------------------------
//  sparse product C = X Y with the oracle's summation order: per output
//  entry from 0.0, contributions in the order of X's row (ascending k)
//--------------------------------------------------------------------------
//  CAP bounds the distinct columns of one output row held in registers /
//  local memory; a row beyond it sets *overflow (the caller then runs the
//  product again with the larger capacity).
template<int CAP>
__global__ void KGemmCount(int nx, const int *__restrict__ xptr, const int *__restrict__ xcol,
                           const int *__restrict__ yptr, const int *__restrict__ ycol,
                           int *__restrict__ cnt, int *__restrict__ overflow)
{
	int lc[CAP];
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x)
	{
		int m = 0;
		bool over = false;
		for(int kx = xptr[i]; kx < xptr[i + 1] && !over; ++kx)
		{
			const int k = xcol[kx];
			for(int ky = yptr[k]; ky < yptr[k + 1]; ++ky)
			{
				const int j = ycol[ky];
				int lo = 0, hi = m;
				while(lo < hi) { const int mid = (lo + hi) >> 1; if(lc[mid] < j) lo = mid + 1; else hi = mid; }
				if(lo < m && lc[lo] == j) continue;
				if(m == CAP) { over = true; break; }
				for(int q = m; q > lo; --q) lc[q] = lc[q - 1];
				lc[lo] = j; ++m;
			}
		}
		if(over) atomicExch(overflow, 1);
		cnt[i] = m;
	}
}

template<int CAP>
__global__ void KGemmFill(int nx, const int *__restrict__ xptr, const int *__restrict__ xcol,
                          const double *__restrict__ xval, const int *__restrict__ yptr,
                          const int *__restrict__ ycol, const double *__restrict__ yval,
                          const int *__restrict__ cptr, int *__restrict__ ccol, double *__restrict__ cval)
{
	int lc[CAP];
	double lv[CAP];
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x)
	{
		int m = 0;
		for(int kx = xptr[i]; kx < xptr[i + 1]; ++kx)
		{
			const int k = xcol[kx];
			const double xv = xval[kx];
			for(int ky = yptr[k]; ky < yptr[k + 1]; ++ky)
			{
				const int j = ycol[ky];
				int lo = 0, hi = m;
				while(lo < hi) { const int mid = (lo + hi) >> 1; if(lc[mid] < j) lo = mid + 1; else hi = mid; }
				if(!(lo < m && lc[lo] == j))
				{
					if(m == CAP) continue;
					for(int q = m; q > lo; --q) { lc[q] = lc[q - 1]; lv[q] = lv[q - 1]; }
					lc[lo] = j; lv[lo] = 0.0; ++m;
				}
				lv[lo] = lv[lo] + xv * yval[ky];
			}
		}
		const int o = cptr[i];
		for(int q = 0; q < m; ++q) { ccol[o + q] = lc[q]; cval[o + q] = lv[q]; }
	}
}

//--------------------------------------------------------------------------
//  The same product with one warp per output row: the row's distinct columns
//  and sums in shared memory (at most CAP), X's row taken entry by entry and
//  each Y row 32 entries at a time (a Y row holds a column once, so the
//  lanes of one step never add into the same sum); every sum gets its
//  contributions in X's row order from 0.0, as the thread-per-row kernels
//  and the oracle give them.  FILL false: the count of every row (a row
//  beyond CAP sets *overflow and is done again by KGemmCount<kRowCap>);
//  FILL true: the row sorted by column into cptr[i]...
//--------------------------------------------------------------------------
template<int CAP, bool FILL>
__global__ void __launch_bounds__(256) KGemmWarp(int nx, const int *__restrict__ xptr, const int *__restrict__ xcol,
                                                 const double *__restrict__ xval, const int *__restrict__ yptr,
                                                 const int *__restrict__ ycol, const double *__restrict__ yval,
                                                 int *__restrict__ cnt, const int *__restrict__ cptr,
                                                 int *__restrict__ ccol, double *__restrict__ cval,
                                                 int *__restrict__ overflow)
{
	constexpr int W = 8;
	__shared__ int scol[W][CAP];
	__shared__ double sval[W][FILL ? CAP : 1];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const unsigned lt = (1u << lane) - 1u;
	const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
	for(long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nx; row += warps)
	{
		const int i = (int)row;
		int m = 0;
		bool over = false;
		const int xe = xptr[i + 1];
		//  X's row 32 entries at a time: each lane loads one entry and its Y
		//  row's bounds, which the warp then takes in order by shuffles
		for(int xb = xptr[i]; xb < xe && !over; xb += 32)
		{
			const int xk = xb + lane;
			const bool av = xk < xe;
			const int kk = av ? xcol[xk] : 0;
			const double xvv = (FILL && av) ? xval[xk] : 0.0;
			const int ys = av ? yptr[kk] : 0, ye = av ? yptr[kk + 1] : 0;
			const int cntx = (xe - xb < 32) ? xe - xb : 32;
		for(int jx = 0; jx < cntx && !over; ++jx)
		{
			const int y0 = __shfl_sync(0xffffffffu, ys, jx);
			const int y1 = __shfl_sync(0xffffffffu, ye, jx);
			const double xv = __shfl_sync(0xffffffffu, xvv, jx);
			for(int base = y0; base < y1 && !over; base += 32)
			{
				const int ky = base + lane;
				const bool active = ky < y1;
				const int j = active ? ycol[ky] : -1;
				int slot = -1;
				if(active)
					for(int q = 0; q < m; ++q) if(scol[w][q] == j) { slot = q; break; }
				const bool need = active && slot < 0;
				const unsigned mask = __ballot_sync(0xffffffffu, need);
				const int add = __popc(mask);
				if(m + add > CAP) { over = true; break; }
				if(need)
				{
					slot = m + __popc(mask & lt);
					scol[w][slot] = j;
					if(FILL) sval[w][slot] = 0.0;
				}
				m += add;
				__syncwarp();
				if(FILL && active) sval[w][slot] = sval[w][slot] + xv * yval[ky];
				__syncwarp();
			}
		}
		}
		if(!FILL)
		{
			if(lane == 0)
			{
				if(over) { atomicExch(overflow, 1); cnt[i] = 0; }
				else cnt[i] = m;
			}
		}
		else
		{
			//  cptr given: the row at its place; else staged at i * CAP with
			//  its count (KGemmCompact moves it once the counts are scanned)
			if(!cptr && lane == 0)
			{
				if(over) { atomicExch(overflow, 1); cnt[i] = 0; }
				else cnt[i] = m;
			}
			const long long o = cptr ? (long long)cptr[i] : (long long)i * CAP;
			for(int q = lane; q < m && !over; q += 32)
			{
				const int c = scol[w][q];
				int r = 0;
				for(int t = 0; t < m; ++t) r += (scol[w][t] < c);
				ccol[o + r] = c;
				cval[o + r] = sval[w][q];
			}
		}
		__syncwarp();
	}
}

//  the staged rows (stride CAP) to their places
template<int CAP>
__global__ void KGemmCompact(int nx, const int *__restrict__ cptr, const int *__restrict__ tcol,
                             const double *__restrict__ tval, int *__restrict__ ccol, double *__restrict__ cval)
{
	for(long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)nx * CAP;
	    e += (long long)gridDim.x * blockDim.x)
	{
		const int i = (int)(e / CAP), r = (int)(e % CAP);
		const int o = cptr[i];
		if(r < cptr[i + 1] - o) { ccol[o + r] = tcol[e]; cval[o + r] = tval[e]; }
	}
}

//--------------------------------------------------------------------------
//  Gauss-Jordan inverse of the coarsest level on [A | I] with partial
//  pivoting (the oracle's GaussJordanInverse, yzo_solver.cpp), blocked.
//  Step k of the unblocked algorithm changes every column j >= k by the same
//  rule, in which only the column's own values, the pivot row p_k, the pivot
//  piv_k and the multipliers f_k(i) = M[src_i][k] (column k before the step,
//  src_i = k for i = p_k, else i) appear:
//      row k:    M[k][j] = M[p][j] / piv
//      row i:    M[i][j] = f == 0 ? M[src_i][j] : M[src_i][j] - f M[k][j]
//  so a panel of B consecutive columns is run through its B steps by one
//  block (recording p, piv and f of each), and every later column then
//  replays those B steps on its own.  Each element sees exactly the
//  operations of the unblocked algorithm, in the same order: the result is
//  the oracle's to the bit, in 2 n / B launches instead of n.
//  M is held column-major (column j at Mc + j n), n <= 3000.
//--------------------------------------------------------------------------
__global__ void KGjInit(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                        const double *__restrict__ val, double *__restrict__ Mc)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		for(int k = ptr[i]; k < ptr[i + 1]; ++k) Mc[(size_t)col[k] * n + i] = val[k];
		Mc[(size_t)(n + i) * n + i] = 1.0;
	}
}

__device__ __forceinline__ void GjBetter(double &best, int &idx, double a, int ia)
{
	if(a > best || (a == best && ia < idx)) { best = a; idx = ia; }
}

//  the pivot of column c of the panel among rows k..n-1: the first row of
//  the largest |a|, taken only when larger than |a_kk| (the sequential
//  rule); the largest |a| (first row among equals) over each warp by
//  shuffles, then over the warps' results -- the same choice as any order of
//  comparison (a NaN is never taken, as in the sequential scan)
__device__ __forceinline__ int GjPivot(const double *colc, int n, int k, double *rv, int *ri)
{
	const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, w = t >> 5;
	double best = -1.0; int idx = n;
	for(int i = k + t; i < n; i += nt) GjBetter(best, idx, fabs(colc[i]), i);
	for(int off = 16; off >= 1; off >>= 1)
	{
		const double a = __shfl_down_sync(0xffffffffu, best, off);
		const int ia = __shfl_down_sync(0xffffffffu, idx, off);
		GjBetter(best, idx, a, ia);
	}
	if(lane == 0) { rv[w] = best; ri[w] = idx; }
	__syncthreads();
	if(w == 0)
	{
		const int nw = nt >> 5;
		best = (lane < nw) ? rv[lane] : -1.0; idx = (lane < nw) ? ri[lane] : n;
		for(int off = 16; off >= 1; off >>= 1)
		{
			const double a = __shfl_down_sync(0xffffffffu, best, off);
			const int ia = __shfl_down_sync(0xffffffffu, idx, off);
			GjBetter(best, idx, a, ia);
		}
		if(lane == 0) { rv[32] = best; ri[32] = idx; }
	}
	__syncthreads();
	const int p = (rv[32] > fabs(colc[k])) ? ri[32] : k;
	__syncthreads();
	return p;
}

//  one block of 512 threads: the B columns k0..k0+B-1, their steps; records
//  pivRow, pivVal and F (B x n) for the columns after them
__global__ void __launch_bounds__(512) KGjPanel(int n, int k0, int B, const double *__restrict__ Mc,
                                                double *__restrict__ F, int *__restrict__ pivRow,
                                                double *__restrict__ pivVal)
{
	extern __shared__ double smem[];
	double *P = smem;                                  // B columns of n
	double *rv = smem + (size_t)B * n;                 // 512 reduction values
	int *ri = reinterpret_cast<int *>(rv + 512);       // 512 reduction indices
	__shared__ double spiv;
	const int t = threadIdx.x, nt = blockDim.x;
	for(int e = t; e < B * n; e += nt) P[e] = Mc[(size_t)k0 * n + e];
	__syncthreads();
	const int lane = t & 31, warp = t >> 5, nw = nt >> 5;
	for(int c = 0; c < B; ++c)
	{
		const int k = k0 + c;
		double *colc = P + (size_t)c * n;
		const int p = GjPivot(colc, n, k, rv, ri);
		if(t == 0) { spiv = colc[p]; pivRow[c] = p; pivVal[c] = colc[p]; }
		//  the multipliers, column c before the step
		for(int i = t; i < n; i += nt) F[(size_t)c * n + i] = colc[(i == p) ? k : i];
		__syncthreads();
		const double piv = spiv;
		//  the step on the panel's columns c..B-1, one warp per column
		for(int cc = c + warp; cc < B; cc += nw)
		{
			double *cl = P + (size_t)cc * n;
			const double colp = cl[p], colk = cl[k];
			__syncwarp();
			const double rowK = colp / piv;
			for(int i = lane; i < n; i += 32)
			{
				double out;
				if(i == k) out = rowK;
				else
				{
					const int src = (i == p) ? k : i;
					const double f = F[(size_t)c * n + i];
					const double mij = (src == k) ? colk : cl[i];
					out = (f == 0.0) ? mij : mij - f * rowK;
				}
				cl[i] = out;
			}
			__syncwarp();
		}
		__syncthreads();
	}
}

//  every column j >= jStart replays the panel's B steps; one block per column
__global__ void KGjUpdate(int n, int k0, int B, int jStart, double *__restrict__ Mc, const double *__restrict__ F,
                          const int *__restrict__ pivRow, const double *__restrict__ pivVal)
{
	extern __shared__ double colv[];
	__shared__ double sColp, sColk;
	const int j = jStart + blockIdx.x;
	const int t = threadIdx.x, nt = blockDim.x;
	double *g = Mc + (size_t)j * n;
	for(int i = t; i < n; i += nt) colv[i] = g[i];
	__syncthreads();
	for(int c = 0; c < B; ++c)
	{
		const int k = k0 + c, p = pivRow[c];
		if(t == 0) { sColp = colv[p]; sColk = colv[k]; }
		__syncthreads();
		const double rowK = sColp / pivVal[c], colk = sColk;
		for(int i = t; i < n; i += nt)
		{
			double out;
			if(i == k) out = rowK;
			else
			{
				const int src = (i == p) ? k : i;
				const double f = F[(size_t)c * n + i];
				const double mij = (src == k) ? colk : colv[i];
				out = (f == 0.0) ? mij : mij - f * rowK;
			}
			colv[i] = out;
		}
		__syncthreads();
	}
	for(int i = t; i < n; i += nt) g[i] = colv[i];
}

//  the right half of [I | A^-1], row-major
__global__ void KGjExtract(int n, const double *__restrict__ Mc, double *__restrict__ inv)
{
	const long long total = (long long)n * n;
	for(long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x)
	{
		const int i = (int)(e / n), j = (int)(e % n);
		inv[(size_t)i * n + j] = Mc[(size_t)(n + j) * n + i];
	}
}

//--------------------------------------------------------------------------
//  V-cycle.  Every kernel of the solve's iteration takes halt, the state
//  word of its BiCGStab run (non-zero once it has stopped), and does nothing
//  when it is set: the iterations are queued ahead of the host's check.
//--------------------------------------------------------------------------
//  The kernels of the cycle are written for the arithmetic T of the cycle's
//  matrices and vectors (double; float in the FP32 V-cycle, whose matrices
//  are the FP64 set-up's rounded to float).  The right-hand side f of the
//  finest level and the result x written there are the Krylov vectors, of
//  type TF and TX: each value is converted to T where it is read and the
//  result to TX where it is written.  With T = TF = TX = double every
//  conversion is the identity and the arithmetic the oracle's.
//--------------------------------------------------------------------------
//  x = m .* f, t = f - A x (x of the neighbours recomputed as m_j * f_j)
template<class T, class TF, class TX>
__global__ void KPreSmoothResidual(const int *__restrict__ halt, int n, const int *__restrict__ ptr,
                                   const int *__restrict__ sellOff, Sten sn, const int *__restrict__ col,
                                   const T *__restrict__ val, const T *__restrict__ M, const TF *__restrict__ f,
                                   TX *__restrict__ x, T *__restrict__ t)
{
	PdlEntry();
	if(halt && *halt) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		int st, len, sd;
		RowRange(ptr, sellOff, i, st, len, sd);
		const T s = RowSumSten(sn, i, st, len, sd, col, val, [&](int c) { return M[c] * (T)f[c]; });
		const T fi = (T)f[i];
		x[i] = (TX)(M[i] * fi);
		t[i] = fi - s;
	}
}

template<class T, class TF, class TX>
__global__ void KPreSmooth(const int *__restrict__ halt, int n, const T *__restrict__ M, const TF *__restrict__ f,
                           TX *__restrict__ x)
{
	PdlEntry();
	if(halt && *halt) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = (TX)(M[i] * (T)f[i]);
}

//  y = A x (from 0.0, stored order)
__global__ void KSpmv(const int *__restrict__ halt, int n, const int *__restrict__ ptr, const int *__restrict__ col,
                      const double *__restrict__ val, const double *__restrict__ x, double *__restrict__ y)
{
	if(halt && *halt) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		y[i] = RowSum(ptr[i], ptr[i + 1] - ptr[i], 1, col, val, [&](int c) { return x[c]; });
}

//  f_c = R t with four lanes per row: lane q sums the row's entries q, q+4,
//  ... from 0.0 and the four partials are folded (p0 + p1) + (p2 + p3) --
//  the oracle's Restrict -- so that the long rows of R (an aggregate and its
//  neighbours) are taken four entries at a time; eight rows a warp, the
//  loop alike for all its lanes
template<class T>
__global__ void KRestrict(const int *__restrict__ halt, int n, const int *__restrict__ ptr, const int *__restrict__ col,
                          const T *__restrict__ val, const T *__restrict__ t, T *__restrict__ y)
{
	PdlEntry();
	if(halt && *halt) return;
	const int lane = threadIdx.x & 31, q = lane & 3;
	const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
	for(long long base = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 8; base < n; base += warps * 8)
	{
		const long long row = base + (lane >> 2);
		const bool active = row < n;
		T p = T(0);
		if(active)
		{
			const int st = ptr[row], len = ptr[row + 1] - st;
			for(int k = q; k < len; k += 4) p = p + val[st + k] * t[col[st + k]];
		}
		p = p + __shfl_down_sync(0xffffffffu, p, 1);
		p = p + __shfl_down_sync(0xffffffffu, p, 2);
		if(active && q == 0) y[row] = p;
	}
}

//  xout = x + P xc
template<class T>
__global__ void KProlong(const int *__restrict__ halt, int n, const int *__restrict__ pptr, const int *__restrict__ pcol,
                         const T *__restrict__ pval, const T *__restrict__ xc, const T *__restrict__ x,
                         T *__restrict__ xout)
{
	PdlEntry();
	if(halt && *halt) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const T s = RowSum(pptr[i], pptr[i + 1] - pptr[i], 1, pcol, pval, [&](int c) { return xc[c]; });
		xout[i] = x[i] + s;
	}
}

//  xout = x + m .* (f - A x)
template<class T, class TF, class TX>
__global__ void KPostSmooth(const int *__restrict__ halt, int n, const int *__restrict__ ptr,
                            const int *__restrict__ sellOff, Sten sn, const int *__restrict__ col,
                            const T *__restrict__ val, const T *__restrict__ M, const TF *__restrict__ f,
                            const T *__restrict__ x, TX *__restrict__ xout)
{
	PdlEntry();
	if(halt && *halt) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		int st, len, sd;
		RowRange(ptr, sellOff, i, st, len, sd);
		const T s = RowSumSten(sn, i, st, len, sd, col, val, [&](int c) { return x[c]; });
		const T t = (T)f[i] - s;
		xout[i] = (TX)(x[i] + M[i] * t);
	}
}

//  x = inv f, inv row-major: one warp per row, lane l sums j = l, l+32, ...
//  from 0.0 (coalesced reads of the row), then a pairwise shuffle fold
template<class T, class TF, class TX>
__global__ void KDenseMV(const int *__restrict__ halt, int n, const T *__restrict__ inv, const TF *__restrict__ f,
                         TX *__restrict__ x)
{
	PdlEntry();
	if(halt && *halt) return;
	const int lane = threadIdx.x & 31;
	const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
	for(long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps)
	{
		const T *row = inv + (size_t)i * n;
		T s = T(0);
		for(int j = lane; j < n; j += 32) s = s + row[j] * (T)f[j];
#pragma unroll
		for(int off = 16; off >= 1; off >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, off);
		if(lane == 0) x[i] = (TX)s;
	}
}

//--------------------------------------------------------------------------
//  The coarse levels of the FP32 cycle with L lanes per row (L = 2, 4, 8):
//  lane q sums the row's entries q, q + L, ... and the group folds its L
//  partials by shuffles.  The coarse rows (an aggregate's Galerkin row, 10
//  to 30 entries) are few, so one thread a row leaves most of the GPU idle;
//  the FP32 cycle's sums are not the oracle's to begin with, so their order
//  is free.  32 / L rows a warp, the loop alike for all its lanes.
//--------------------------------------------------------------------------
template<int L, class T, class XF>
__device__ __forceinline__ T RowSumLanes(const int *__restrict__ ptr, const int *__restrict__ col,
                                         const T *__restrict__ val, long long row, bool active, int q, XF xf)
{
	T p = T(0);
	if(active)
	{
		const int st = ptr[row], len = ptr[row + 1] - st;
		for(int k = q; k < len; k += L) p = p + val[st + k] * xf(col[st + k]);
	}
#pragma unroll
	for(int off = L / 2; off >= 1; off >>= 1) p = p + __shfl_down_sync(0xffffffffu, p, off);
	return p;
}

#define YZ_LANE_LOOP(L)                                                                              \
	const int lane_ = threadIdx.x & 31, q = lane_ % (L);                                             \
	const long long warps_ = ((long long)gridDim.x * blockDim.x) >> 5;                              \
	for(long long base_ = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32 / (L));   \
	    base_ < n; base_ += warps_ * (32 / (L)))

//  x = m .* f, t = f - A x
template<int L, class T>
__global__ void KPreSmoothResidualL(const int *__restrict__ halt, int n, const int *__restrict__ ptr,
                                    const int *__restrict__ col, const T *__restrict__ val, const T *__restrict__ M,
                                    const T *__restrict__ f, T *__restrict__ x, T *__restrict__ t)
{
	PdlEntry();
	if(halt && *halt) return;
	YZ_LANE_LOOP(L)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < n;
		const T s = RowSumLanes<L>(ptr, col, val, row, active, q, [&](int c) { return M[c] * f[c]; });
		if(active && q == 0)
		{
			const T fi = f[row];
			x[row] = M[row] * fi;
			t[row] = fi - s;
		}
	}
}

//  xout = x + m .* (f - A x)
template<int L, class T>
__global__ void KPostSmoothL(const int *__restrict__ halt, int n, const int *__restrict__ ptr,
                             const int *__restrict__ col, const T *__restrict__ val, const T *__restrict__ M,
                             const T *__restrict__ f, const T *__restrict__ x, T *__restrict__ xout)
{
	PdlEntry();
	if(halt && *halt) return;
	YZ_LANE_LOOP(L)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < n;
		const T s = RowSumLanes<L>(ptr, col, val, row, active, q, [&](int c) { return x[c]; });
		if(active && q == 0) xout[row] = x[row] + M[row] * (f[row] - s);
	}
}

//  xout = x + P xc
template<int L, class T>
__global__ void KProlongL(const int *__restrict__ halt, int n, const int *__restrict__ pptr, const int *__restrict__ pcol,
                          const T *__restrict__ pval, const T *__restrict__ xc, const T *__restrict__ x,
                          T *__restrict__ xout)
{
	PdlEntry();
	if(halt && *halt) return;
	YZ_LANE_LOOP(L)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < n;
		const T s = RowSumLanes<L>(pptr, pcol, pval, row, active, q, [&](int c) { return xc[c]; });
		if(active && q == 0) xout[row] = x[row] + s;
	}
}

//--------------------------------------------------------------------------
//  A coarse level's way down and way up, each in one launch.  Below the
//  finest level the V-cycle's phases are short (a few thousand rows) and
//  each costs a kernel boundary more than its work; two of the four per
//  level go by recomputing what the separate kernels passed through memory:
//
//    down:  fc = R (f - A (m .* f))              (pre-smoothing from zero,
//           the residual and the restriction; t_j recomputed by every R row
//           that holds j)
//    up:    x = xt + m .* (f - A xt),  xt = m .* f + P xc
//           (prolongation and post-smoothing; xt_k recomputed by every row
//           whose A row holds k)
//
//  The same arithmetic as the separate kernels in another order: the FP32
//  cycle's sums are not the oracle's.  L lanes a row (the down kernel's rows
//  are the next level's), each lane a fixed share of the row's entries, the
//  partials folded by shuffles: deterministic.
//--------------------------------------------------------------------------
template<int L, class T>
__global__ void KDownFused(const int *__restrict__ halt, int n, const int *__restrict__ rptr,
                           const int *__restrict__ rcol, const T *__restrict__ rval, const int *__restrict__ ptr,
                           const int *__restrict__ col, const T *__restrict__ val, const T *__restrict__ M,
                           const T *__restrict__ f, T *__restrict__ fc)
{
	PdlEntry();
	if(halt && *halt) return;
	YZ_LANE_LOOP(L)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < n;
		const T s = RowSumLanes<L>(rptr, rcol, rval, row, active, q, [&](int j) {
			T a = T(0);
			const int st = ptr[j], en = ptr[j + 1];
			for(int e = st; e < en; ++e)
			{
				const int c = col[e];
				a = a + val[e] * (M[c] * f[c]);
			}
			return f[j] - a;
		});
		if(active && q == 0) fc[row] = s;
	}
}

template<int L, class T>
__global__ void KUpFused(const int *__restrict__ halt, int n, const int *__restrict__ ptr, const int *__restrict__ col,
                         const T *__restrict__ val, const T *__restrict__ M, const int *__restrict__ pptr,
                         const int *__restrict__ pcol, const T *__restrict__ pval, const T *__restrict__ f,
                         const T *__restrict__ xc, T *__restrict__ x)
{
	PdlEntry();
	if(halt && *halt) return;
	auto xt = [&](int k) {
		T s = T(0);
		for(int e = pptr[k], en = pptr[k + 1]; e < en; ++e) s = s + pval[e] * xc[pcol[e]];
		return M[k] * f[k] + s;
	};
	YZ_LANE_LOOP(L)
	{
		const long long row = base_ + lane_ / L;
		const bool active = row < n;
		const T s = RowSumLanes<L>(ptr, col, val, row, active, q, xt);
		if(active && q == 0) x[row] = xt((int)row) + M[row] * (f[row] - s);
	}
}
#undef YZ_LANE_LOOP

//  the FP32 copies of the V-cycle's matrices: dst_k[i] = (float)src_k[i] over
//  a list of arrays, one launch for all of them
struct RoundList
{
	enum { kMax = 64 };
	const double *src[kMax];
	float *dst[kMax];
	long long n[kMax];
	int count;
};

__global__ void KRoundToFloat(RoundList L)
{
	const long long stride = (long long)gridDim.x * blockDim.x;
	for(int k = 0; k < L.count; ++k)
	{
		const double *__restrict__ s = L.src[k];
		float *__restrict__ d = L.dst[k];
		for(long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L.n[k]; i += stride) d[i] = (float)s[i];
	}
}

__global__ void KDiagApply(const int *__restrict__ halt, int n, const double *__restrict__ M, const double *__restrict__ r, double *__restrict__ z)
{
	if(halt && *halt) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = M[i] * r[i];
}

} // namespace yz
