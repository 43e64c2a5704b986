// yz_unet.cu -- the learned preconditioner's network on the device: the
// 3x3 convolution as an implicit GEMM on the tensor cores (tcgen05.mma,
// BF16 operands staged in shared memory, FP32 accumulator in TMEM), the
// pooling, upsampling and skip kernels, the loss, the backward pass
// (transposed convolutions on the same tensor-core kernel, weight gradients
// on the CUDA cores with a fixed summation order), Adam, and the sample ring
// the solver fills with (residual, AMG correction) pairs.  The layout and
// the architecture are described in yz_learned.h.
#include "yz_learned.h"
#include "yz_tc.cuh"

#include <algorithm>
#include <cmath>
#include <random>

namespace yz {

using bf16 = __nv_bfloat16;

namespace {

constexpr int kTile = 128;                    // pixels per CTA (the MMA's M)
constexpr int kHalo = kTile + 2;              // pixels of one halo row
constexpr long long kWaitBudget = 2000000000LL;   // clock cycles an mbarrier wait may take (~1 s)
constexpr int kConvSmemMax = 200 * 1024;      // dynamic shared memory of the convolution kernel

//==========================================================================
//  The 3x3 convolution, one CTA of 128 threads per 128 consecutive pixels.
//
//  y[p][coff + n] = act(bias[n] + sum_{tap, ci} x[p + dy W + dx][ci] w[n][tap][ci])
//
//  A (128 pixels x K) is never formed: the three halo rows of the tile --
//  pixels p0 + dy W - 1 .. p0 + dy W + 128 for dy = -1, 0, 1, every channel --
//  are staged once in shared memory as 8-channel chunks of 130 rows of 16
//  bytes, and the A operand of tap (dy, dx) is the descriptor of that buffer
//  started dx + 1 rows in.  B (the tap's weights, N rows of 8 channels per
//  chunk) is staged per group of taps that fits beside A.  One thread issues
//  the MMAs (M = 128, N, K = 16 per instruction) into one TMEM accumulator;
//  four warps read it back, each its 32 lanes (pixels), and write bf16.
//==========================================================================
struct ConvArgs
{
	const bf16 *x;
	bf16 *y;
	const bf16 *w;         // [9][cin/8][n][8]
	const float *bias;     // [n] or null
	int H, W, cin, n, ldy, coff, realW, realH, relu, tpg;
	const int *halt;
	int *err;
};

__host__ __device__ inline int ConvAStride(int cin) { return (cin / 8) * kHalo * 16; }

size_t ConvSmem(int cin, int n, int tpg) { return (size_t)3 * ConvAStride(cin) + (size_t)tpg * (cin / 8) * n * 16 + 64; }

int ConvTapsPerGroup(int cin, int n)
{
	const long long perTap = (long long)(cin / 8) * n * 16;
	const long long budget = (long long)kConvSmemMax - 3LL * ConvAStride(cin) - 64;
	long long t = budget / perTap;
	if(t > 9) t = 9;
	if(t < 1) throw UsageError("conv: a tap's weights do not fit in shared memory");
	return (int)t;
}

__global__ void __launch_bounds__(128) KConv3x3(ConvArgs a)
{
	if(a.halt && *a.halt != 0) return;
	extern __shared__ __align__(1024) unsigned char smem[];
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int chunks = a.cin >> 3;
	const int aStride = chunks * kHalo * 16;
	unsigned char *As = smem;
	unsigned char *Bs = smem + 3 * aStride;
	const int bPerTap = chunks * a.n;                       // 16-byte rows per tap
	uint64_t *bar = reinterpret_cast<uint64_t *>(Bs + (size_t)a.tpg * bPerTap * 16);
	uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
	const uint32_t ncols = a.n <= 32 ? 32u : (a.n <= 64 ? 64u : (a.n <= 128 ? 128u : 256u));
	const int HW = a.H * a.W;
	const int p0 = blockIdx.x * kTile;

	if(warp == 0) tc::TmemAlloc(slot, ncols);
	if(tid == 0) tc::BarInit(bar, 1);
	{
		const int per = kHalo * chunks;
		for(int idx = tid; idx < 3 * per; idx += blockDim.x)
		{
			const int dyi = idx / per, rem = idx - dyi * per;
			const int px = rem / chunks, c = rem - px * chunks;
			const long long q = (long long)p0 + (long long)(dyi - 1) * a.W + (px - 1);
			const bool in = q >= 0 && q < HW;
			tc::CpAsync16(As + dyi * aStride + c * (kHalo * 16) + px * 16,
			              a.x + (in ? (size_t)q * a.cin + c * 8 : (size_t)0), in);
		}
	}
	tc::CpAsyncWaitAll();
	tc::FenceBeforeSync();
	__syncthreads();
	tc::FenceAfterSync();
	const uint32_t tmem = *slot;
	const uint32_t idesc = tc::IdescBf16(kTile, a.n);
	bool ok = true;
	uint32_t phase = 0;
	bool first = true;
	for(int t0 = 0; t0 < 9; t0 += a.tpg)
	{
		const int tg = min(a.tpg, 9 - t0);
		const uint4 *src = reinterpret_cast<const uint4 *>(a.w) + (size_t)t0 * bPerTap;
		for(int idx = tid; idx < tg * bPerTap; idx += blockDim.x)
			tc::CpAsync16(reinterpret_cast<uint4 *>(Bs) + idx, src + idx, true);
		tc::CpAsyncWaitAll();
		tc::FenceProxyAsync();
		__syncthreads();
		if(tid == 0)
		{
			tc::FenceAfterSync();
			const uint32_t aBase = tc::SmemAddr(As), bBase = tc::SmemAddr(Bs);
			for(int t = t0; t < t0 + tg; ++t)
			{
				const int dyi = t / 3, dxi = t - 3 * dyi;
				for(int j = 0; j < chunks; j += 2)
				{
					const uint64_t ad = tc::SmemDesc(aBase + dyi * aStride + j * (kHalo * 16) + dxi * 16, kHalo * 16, 128);
					const uint64_t bd = tc::SmemDesc(bBase + ((t - t0) * chunks + j) * a.n * 16, a.n * 16, 128);
					tc::MmaBf16(tmem, ad, bd, idesc, first ? 0u : 1u);
					first = false;
				}
			}
			tc::Commit(bar);
		}
		const bool mine = tc::BarWait(bar, phase, kWaitBudget);
		phase ^= 1u;
		//  every thread takes the same path from here
		if(__syncthreads_or(mine ? 0 : 1)) { ok = false; break; }
	}
	tc::FenceAfterSync();
	if(ok)
	{
		const int m = warp * 32 + lane;
		const int p = p0 + m;
		const uint32_t lanes = tmem + ((uint32_t)(warp * 32) << 16);
		bool real = false;
		if(p < HW)
		{
			const int py = p / a.W, px = p - py * a.W;
			real = (px < a.realW && py < a.realH);
		}
		for(int cb = 0; cb < a.n; cb += 16)
		{
			float v[16];
			tc::TmemLoad16(lanes + (uint32_t)cb, v);
			if(p < HW)
			{
				__align__(16) bf16 o[16];
#pragma unroll
				for(int e = 0; e < 16; ++e)
				{
					float t = v[e];
					if(a.bias) t = t + a.bias[cb + e];
					if(a.relu) t = fmaxf(t, 0.0f);
					o[e] = __float2bfloat16_rn(real ? t : 0.0f);
				}
				uint4 *dst = reinterpret_cast<uint4 *>(a.y + (size_t)p * a.ldy + a.coff + cb);
				dst[0] = reinterpret_cast<const uint4 *>(o)[0];
				dst[1] = reinterpret_cast<const uint4 *>(o)[1];
			}
		}
	}
	else if(tid == 0)
		atomicExch(a.err, 1);
	tc::FenceBeforeSync();
	__syncthreads();
	if(warp == 0)
	{
		tc::FenceAfterSync();
		tc::TmemDealloc(tmem, ncols);
	}
}

//==========================================================================
//  element-wise kernels (one thread per pixel and 8-channel group)
//==========================================================================
struct Lv
{
	int H, W, realH, realW;
};

__device__ __forceinline__ bool IsReal(const Lv &l, int p, int &y, int &x)
{
	y = p / l.W;
	x = p - y * l.W;
	return x < l.realW && y < l.realH;
}

__device__ __forceinline__ void Load8(const bf16 *s, float (&v)[8])
{
	const uint4 u = *reinterpret_cast<const uint4 *>(s);
	const bf16 *b = reinterpret_cast<const bf16 *>(&u);
#pragma unroll
	for(int e = 0; e < 8; ++e) v[e] = __bfloat162float(b[e]);
}

__device__ __forceinline__ void Store8(bf16 *d, const float (&v)[8])
{
	__align__(16) bf16 b[8];
#pragma unroll
	for(int e = 0; e < 8; ++e) b[e] = __float2bfloat16_rn(v[e]);
	*reinterpret_cast<uint4 *>(d) = *reinterpret_cast<const uint4 *>(b);
}

//  2x2 average of channels [0, C) of src (stride cs) into dst (C channels)
__global__ void KPool(int C, int cs, const bf16 *__restrict__ src, Lv ls, bf16 *__restrict__ dst, Lv ld, const int *halt)
{
	if(halt && *halt != 0) return;
	const int g = C / 8;
	const long long total = (long long)ld.H * ld.W * g;
	for(long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
	{
		const int q = (int)(k / g), c = (int)(k - (long long)q * g) * 8;
		int y, x;
		float o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		if(IsReal(ld, q, y, x))
		{
			float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
			for(int j = 0; j < 4; ++j)
			{
				const int p = (2 * y + (j >> 1)) * ls.W + 2 * x + (j & 1);
				float v[8];
				Load8(src + (size_t)p * cs + c, v);
#pragma unroll
				for(int e = 0; e < 8; ++e) s[e] = s[e] + v[e];
			}
#pragma unroll
			for(int e = 0; e < 8; ++e) o[e] = 0.25f * s[e];
		}
		Store8(dst + (size_t)q * C + c, o);
	}
}

//  nearest upsampling of src (C channels, level l+1) into channels
//  [coff, coff + C) of dst (stride cs, level l)
__global__ void KUp(int C, const bf16 *__restrict__ src, Lv ls, bf16 *__restrict__ dst, int cs, int coff, Lv ld,
                    const int *halt)
{
	if(halt && *halt != 0) return;
	const int g = C / 8;
	const long long total = (long long)ld.H * ld.W * g;
	for(long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
	{
		const int p = (int)(k / g), c = (int)(k - (long long)p * g) * 8;
		int y, x;
		float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		if(IsReal(ld, p, y, x)) Load8(src + ((size_t)(y >> 1) * ls.W + (x >> 1)) * C + c, v);
		Store8(dst + (size_t)p * cs + coff + c, v);
	}
}

//  the gradient of an upsampled tensor: the sum over the four children of
//  channels [coff, coff + C) of gU (stride cs, level l), where the forward
//  activation D (level l+1, after ReLU) is positive
__global__ void KUpBack(int C, const bf16 *__restrict__ gU, int cs, int coff, Lv lh, const bf16 *__restrict__ D,
                        Lv ll, bf16 *__restrict__ gD, int act)
{
	const int g = C / 8;
	const long long total = (long long)ll.H * ll.W * g;
	for(long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
	{
		const int q = (int)(k / g), c = (int)(k - (long long)q * g) * 8;
		int y, x;
		float o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		if(IsReal(ll, q, y, x))
		{
			float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
			for(int j = 0; j < 4; ++j)
			{
				const int cy = 2 * y + (j >> 1), cx = 2 * x + (j & 1);
				if(cx >= lh.realW || cy >= lh.realH) continue;
				float v[8];
				Load8(gU + ((size_t)cy * lh.W + cx) * cs + coff + c, v);
#pragma unroll
				for(int e = 0; e < 8; ++e) s[e] = s[e] + v[e];
			}
			float d[8];
			Load8(D + (size_t)q * C + c, d);
#pragma unroll
			for(int e = 0; e < 8; ++e) o[e] = (!act || d[e] > 0.0f) ? s[e] : 0.0f;
		}
		Store8(gD + (size_t)q * C + c, o);
	}
}

//  the gradient of an encoder output E (channels [0, C) of U, stride cs,
//  level l): its skip part from gU plus a quarter of the pooled gradient gP
//  (level l+1) of its parent, where E is positive
__global__ void KSkipBack(int C, const bf16 *__restrict__ gU, const bf16 *__restrict__ U, int cs, Lv lh,
                          const bf16 *__restrict__ gP, Lv ll, bf16 *__restrict__ gE, int act)
{
	const int g = C / 8;
	const long long total = (long long)lh.H * lh.W * g;
	for(long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x)
	{
		const int p = (int)(k / g), c = (int)(k - (long long)p * g) * 8;
		int y, x;
		float o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		if(IsReal(lh, p, y, x))
		{
			float a[8], b[8], e8[8];
			Load8(gU + (size_t)p * cs + c, a);
			Load8(gP + ((size_t)(y >> 1) * ll.W + (x >> 1)) * C + c, b);
			Load8(U + (size_t)p * cs + c, e8);
#pragma unroll
			for(int e = 0; e < 8; ++e) o[e] = (!act || e8[e] > 0.0f) ? a[e] + 0.25f * b[e] : 0.0f;
		}
		Store8(gE + (size_t)p * C + c, o);
	}
}

//==========================================================================
//  features, output, samples
//==========================================================================
//  sum of r^2 by the fixed tree; rms = sqrt(sum / n), inv = 1 / rms
__global__ void __launch_bounds__(kRT) KSumSq(int n, const double *__restrict__ r, RedScratch rs, double *rms,
                                             float *inv, const int *halt)
{
	if(halt && *halt != 0) return;
	__shared__ double sh[kRT];
	double a[1] = {0.0};
	const int i = blockIdx.x * kRT + threadIdx.x;
	if(i < n) a[0] = r[i] * r[i];
	double tot[1];
	if(GridFold<1>(a, sh, rs, tot) && threadIdx.x == 0)
	{
		const double v = sqrt(tot[0] / (double)n);
		*rms = v;
		*inv = v > 0.0 ? (float)(1.0 / v) : 0.0f;
	}
}

//  the diagonal and height features of the rows
__global__ void KAux(int n, const double *__restrict__ vals, const int *__restrict__ rowptr,
                     const double *__restrict__ h, float *__restrict__ aux)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const double d = fabs(vals[rowptr[i]]);
		aux[i] = (float)(log10(d > 1e-30 ? d : 1e-30) * 0.25);
		float fh = 0.0f;
		if(h)
		{
			const double hv = h[i];
			fh = (float)(log10(hv > 1e-30 ? hv : 1e-30) * 0.5 + 1.0);
		}
		aux[n + i] = fh;
	}
}

//  The input channels of a pixel: the residual r (normalised) and its
//  products with the two features and their squares and product -- every
//  channel linear in r, so that without activations the network is a linear
//  operator on r whose coefficients vary with the matrix diagonal and the
//  film height
__device__ __forceinline__ void InputChannels(float r, float f1, float f2, float (&v)[8])
{
	v[0] = r;
	v[1] = r * f1;
	v[2] = r * f2;
	v[3] = (r * f1) * f1;
	v[4] = (r * f2) * f2;
	v[5] = (r * f1) * f2;
	v[6] = 0.0f;
	v[7] = 0.0f;
}

//  the input image: channels 0..5 of InputChannels, 6..15 zero
__global__ void KPackF(int n, int nx, Lv l0, const double *__restrict__ r, const float *__restrict__ inv,
                       const float *__restrict__ aux, bf16 *__restrict__ F, const int *halt)
{
	if(halt && *halt != 0) return;
	const int HW = l0.H * l0.W;
	const float s = *inv;
	for(int p = blockIdx.x * blockDim.x + threadIdx.x; p < HW; p += gridDim.x * blockDim.x)
	{
		int y, x;
		float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		if(IsReal(l0, p, y, x))
		{
			const int i = y * nx + x;
			InputChannels((float)r[i] * s, aux[i], aux[n + i], v);
		}
		const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		Store8(F + (size_t)p * 16, v);
		Store8(F + (size_t)p * 16 + 8, zero);
	}
}

//  z_i = rms s (b + sum_c w_c D0[p(i)][c]), s the training targets' scale
__global__ void KOut(int n, int nx, Lv l0, const bf16 *__restrict__ D0, const float *__restrict__ w, const float *b,
                     const double *__restrict__ rms, const float *__restrict__ tsc, double *__restrict__ z,
                     const int *halt)
{
	if(halt && *halt != 0) return;
	const double sc = *rms * (double)*tsc;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const int y = i / nx, x = i - y * nx;
		const size_t p = (size_t)y * l0.W + x;
		float v0[8], v1[8];
		Load8(D0 + p * 16, v0);
		Load8(D0 + p * 16 + 8, v1);
		float s = *b;
#pragma unroll
		for(int c = 0; c < 8; ++c) s = s + w[c] * v0[c];
#pragma unroll
		for(int c = 0; c < 8; ++c) s = s + w[8 + c] * v1[c];
		z[i] = sc * (double)s;
	}
}

//  a training pair into ring slot s: r / rms, z / rms, the two features
__global__ void KStoreSample(int n, const double *__restrict__ r, const double *__restrict__ z,
                             const float *__restrict__ inv, const float *__restrict__ aux, float *__restrict__ slot,
                             int *valid, const int *halt)
{
	const bool off = halt && *halt != 0;
	if(blockIdx.x == 0 && threadIdx.x == 0) *valid = off ? 0 : 1;
	if(off) return;
	const float s = *inv;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		slot[i] = (float)r[i] * s;
		slot[n + i] = (float)z[i] * s;
		slot[2 * n + i] = aux[i];
		slot[3 * n + i] = aux[n + i];
	}
}

//  the input image and the target map of a stored pair
__global__ void KBuildImage(int n, int nx, Lv l0, const float *__restrict__ slot, const float *__restrict__ tsc,
                            bf16 *__restrict__ F, float *__restrict__ T)
{
	const int HW = l0.H * l0.W;
	const float inv = 1.0f / *tsc;
	for(int p = blockIdx.x * blockDim.x + threadIdx.x; p < HW; p += gridDim.x * blockDim.x)
	{
		int y, x;
		float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		float t = 0.0f;
		if(IsReal(l0, p, y, x))
		{
			const int i = y * nx + x;
			InputChannels(slot[i], slot[2 * n + i], slot[3 * n + i], v);
			t = slot[n + i] * inv;
		}
		const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
		Store8(F + (size_t)p * 16, v);
		Store8(F + (size_t)p * 16 + 8, zero);
		T[p] = t;
	}
}

//  sum of z^2 over a stored pair's target, per block (the training set's
//  target scale)
__global__ void __launch_bounds__(kRT) KSlotSq(int n, const float *__restrict__ z, float *__restrict__ part)
{
	__shared__ double sh[kRT];
	double a[1] = {0.0};
	const int i = blockIdx.x * kRT + threadIdx.x;
	if(i < n) a[0] = (double)z[i] * (double)z[i];
	BlockTree<1>(a, sh);
	if(threadIdx.x == 0) part[blockIdx.x] = (float)a[0];
}

//  The loss over the real pixels, L = sum (out - t)^2 / n, and its
//  gradient: dL/dD0 (where D0 > 0) as bf16, and per block the partials of
//  L, dL/dw_c (16) and dL/db in a fixed order (BlockTree)
constexpr int kLossQ = 18;
__global__ void __launch_bounds__(kRT) KLoss(int n, Lv l0, const bf16 *__restrict__ D0, const float *__restrict__ T,
                                            const float *__restrict__ w, const float *b, bf16 *__restrict__ gD0,
                                            float *__restrict__ part, int act)
{
	__shared__ double sh[kLossQ * kRT];
	double a[kLossQ];
#pragma unroll
	for(int q = 0; q < kLossQ; ++q) a[q] = 0.0;
	const int p = blockIdx.x * kRT + threadIdx.x;
	const int HW = l0.H * l0.W;
	if(p < HW)
	{
		int y, x;
		float g[16];
#pragma unroll
		for(int c = 0; c < 16; ++c) g[c] = 0.0f;
		if(IsReal(l0, p, y, x))
		{
			float v0[8], v1[8];
			Load8(D0 + (size_t)p * 16, v0);
			Load8(D0 + (size_t)p * 16 + 8, v1);
			float d[16];
#pragma unroll
			for(int c = 0; c < 8; ++c) { d[c] = v0[c]; d[8 + c] = v1[c]; }
			float s = *b;
#pragma unroll
			for(int c = 0; c < 16; ++c) s = s + w[c] * d[c];
			const float diff = s - T[p];
			const float gr = 2.0f * diff / (float)n;
			a[0] = (double)diff * (double)diff / (double)n;
#pragma unroll
			for(int c = 0; c < 16; ++c)
			{
				a[1 + c] = (double)gr * (double)d[c];
				g[c] = (!act || d[c] > 0.0f) ? gr * w[c] : 0.0f;
			}
			a[17] = (double)gr;
		}
		float g0[8], g1[8];
#pragma unroll
		for(int c = 0; c < 8; ++c) { g0[c] = g[c]; g1[c] = g[8 + c]; }
		Store8(gD0 + (size_t)p * 16, g0);
		Store8(gD0 + (size_t)p * 16 + 8, g1);
	}
	BlockTree<kLossQ>(a, sh);
	if(threadIdx.x == 0)
	{
#pragma unroll
		for(int q = 0; q < kLossQ; ++q) part[(size_t)blockIdx.x * kLossQ + q] = (float)a[q];
	}
}

//  the loss partials summed in block order; the output layer's gradient
//  added to grad, the loss to out[0]
__global__ void KLossReduce(int nb, const float *__restrict__ part, double *out, float *grad, size_t wOff, size_t bOff,
                            int bias)
{
	const int q = threadIdx.x;
	if(q >= kLossQ) return;
	double s = 0.0;
	for(int b = 0; b < nb; ++b) s = s + (double)part[(size_t)b * kLossQ + q];
	if(q == 0) out[0] = out[0] + s;
	else if(q < 17) grad[wOff + q - 1] = grad[wOff + q - 1] + (float)s;
	else if(bias) grad[bOff] = grad[bOff] + (float)s;
}

//  per-sample relative error parts: |out - t|^2 and |t|^2 over the real pixels
__global__ void __launch_bounds__(kRT) KValErr(Lv l0, const bf16 *__restrict__ D0, const float *__restrict__ T,
                                              const float *__restrict__ w, const float *b, float *__restrict__ part)
{
	__shared__ double sh[2 * kRT];
	double a[2] = {0.0, 0.0};
	const int p = blockIdx.x * kRT + threadIdx.x;
	int y, x;
	if(p < l0.H * l0.W && IsReal(l0, p, y, x))
	{
		float v0[8], v1[8];
		Load8(D0 + (size_t)p * 16, v0);
		Load8(D0 + (size_t)p * 16 + 8, v1);
		float s = *b;
#pragma unroll
		for(int c = 0; c < 8; ++c) s = s + w[c] * v0[c];
#pragma unroll
		for(int c = 0; c < 8; ++c) s = s + w[8 + c] * v1[c];
		const double d = (double)s - (double)T[p];
		a[0] = d * d;
		a[1] = (double)T[p] * (double)T[p];
	}
	BlockTree<2>(a, sh);
	if(threadIdx.x == 0) { part[2 * blockIdx.x] = (float)a[0]; part[2 * blockIdx.x + 1] = (float)a[1]; }
}

__global__ void KOutMap(int n, int nx, Lv l0, const bf16 *__restrict__ D0, const float *__restrict__ w, const float *b,
                        float *__restrict__ out)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const int y = i / nx, x = i - y * nx;
		const size_t p = (size_t)y * l0.W + x;
		float v0[8], v1[8];
		Load8(D0 + p * 16, v0);
		Load8(D0 + p * 16 + 8, v1);
		float s = *b;
#pragma unroll
		for(int c = 0; c < 8; ++c) s = s + w[c] * v0[c];
#pragma unroll
		for(int c = 0; c < 8; ++c) s = s + w[8 + c] * v1[c];
		out[i] = s;
	}
}

//==========================================================================
//  weight gradients (CUDA cores): block (b, tap) sums
//  dy[p][n] x[p + dy W + dx][ci] over its pixels [b PB, (b+1) PB) in
//  pixel order, 32 pixels at a time through shared memory; the partials of
//  the blocks are summed in block order by KWReduce
//==========================================================================
constexpr int kWgJ = 32;
constexpr int kWgTiles = 2;      // 4 x 4 output tiles per thread (n x cin <= 8192)

__global__ void __launch_bounds__(256) KWGrad(int H, int W, int cin, int n, int pb, const bf16 *__restrict__ x,
                                              const bf16 *__restrict__ dy, float *__restrict__ part,
                                              float *__restrict__ partB)
{
	__shared__ __align__(16) float sx[kWgJ * 128];
	__shared__ __align__(16) float sd[kWgJ * 128];
	const int tap = blockIdx.y;
	const int ody = tap / 3 - 1, odx = tap % 3 - 1;
	const int HW = H * W;
	const int pBeg = blockIdx.x * pb;
	const int pEnd = min(HW, pBeg + pb);
	const int outs = n * cin;
	const int tcs = cin / 4, tiles = (n / 4) * tcs;
	float acc[kWgTiles][16];
#pragma unroll
	for(int k = 0; k < kWgTiles; ++k)
#pragma unroll
		for(int e = 0; e < 16; ++e) acc[k][e] = 0.0f;
	float accB = 0.0f;
	for(int base = pBeg; base < pEnd; base += kWgJ)
	{
		for(int idx = threadIdx.x; idx < kWgJ * n; idx += blockDim.x)
		{
			const int j = idx / n, c = idx - j * n;
			const int p = base + j;
			sd[idx] = (p < pEnd) ? __bfloat162float(dy[(size_t)p * n + c]) : 0.0f;
		}
		for(int idx = threadIdx.x; idx < kWgJ * cin; idx += blockDim.x)
		{
			const int j = idx / cin, c = idx - j * cin;
			const int p = base + j;
			const long long q = (long long)p + (long long)ody * W + odx;
			sx[idx] = (p < pEnd && q >= 0 && q < HW) ? __bfloat162float(x[(size_t)q * cin + c]) : 0.0f;
		}
		__syncthreads();
#pragma unroll
		for(int k = 0; k < kWgTiles; ++k)
		{
			const int t = threadIdx.x + k * blockDim.x;
			if(t < tiles)
			{
				const int n0 = (t / tcs) * 4, c0 = (t - (t / tcs) * tcs) * 4;
				for(int j = 0; j < kWgJ; ++j)
				{
					const float4 av = *reinterpret_cast<const float4 *>(&sd[j * n + n0]);
					const float4 bv = *reinterpret_cast<const float4 *>(&sx[j * cin + c0]);
					const float ar[4] = {av.x, av.y, av.z, av.w}, br[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
					for(int u = 0; u < 4; ++u)
#pragma unroll
						for(int v = 0; v < 4; ++v) acc[k][u * 4 + v] = acc[k][u * 4 + v] + ar[u] * br[v];
				}
			}
		}
		if(tap == 0 && threadIdx.x < n)
			for(int j = 0; j < kWgJ; ++j) accB = accB + sd[j * n + threadIdx.x];
		__syncthreads();
	}
#pragma unroll
	for(int k = 0; k < kWgTiles; ++k)
	{
		const int t = threadIdx.x + k * blockDim.x;
		if(t < tiles)
		{
			const int n0 = (t / tcs) * 4, c0 = (t - (t / tcs) * tcs) * 4;
			float *dst = part + ((size_t)blockIdx.x * 9 + tap) * outs;
#pragma unroll
			for(int u = 0; u < 4; ++u)
#pragma unroll
				for(int v = 0; v < 4; ++v) dst[(n0 + u) * cin + c0 + v] = acc[k][u * 4 + v];
		}
	}
	if(tap == 0 && threadIdx.x < n) partB[(size_t)blockIdx.x * n + threadIdx.x] = accB;
}

//  grad W[n][tap][ci] += sum_b part[b][tap][n][ci]; grad b[n] += sum_b partB[b][n]
__global__ void KWReduce(int nb, int cin, int n, const float *__restrict__ part, const float *__restrict__ partB,
                         float *__restrict__ grad, size_t wOff, size_t bOff, int bias)
{
	const int outs = n * cin;
	const int total = 9 * outs + n;
	for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x)
	{
		if(k < 9 * outs)
		{
			const int tap = k / outs, o = k - tap * outs;
			const int nn = o / cin, ci = o - nn * cin;
			float s = 0.0f;
			for(int b = 0; b < nb; ++b) s = s + part[((size_t)b * 9 + tap) * outs + o];
			const size_t g = wOff + ((size_t)nn * 9 + tap) * cin + ci;
			grad[g] = grad[g] + s;
		}
		else if(bias)
		{
			const int nn = k - 9 * outs;
			float s = 0.0f;
			for(int b = 0; b < nb; ++b) s = s + partB[(size_t)b * n + nn];
			grad[bOff + nn] = grad[bOff + nn] + s;
		}
	}
}

//==========================================================================
//  optimiser and weight packing
//==========================================================================
__global__ void KAdam(size_t np, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                      float *__restrict__ v, float lr, float scale, float c1, float c2)
{
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
	for(size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < np; k += (size_t)gridDim.x * blockDim.x)
	{
		const float gk = g[k] * scale;
		const float mk = b1 * m[k] + (1.0f - b1) * gk;
		const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
		m[k] = mk;
		v[k] = vk;
		p[k] = p[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
	}
}

//  wf[tap][cin/8][n][8] = W[n][tap][ci]; wb (the transposed convolution,
//  cin' = n, n' = cin)[tap'][n/8][cin][8] = W[n][8 - tap'][ci]
__global__ void KPackW(int cin, int n, const float *__restrict__ W, bf16 *__restrict__ wf, bf16 *__restrict__ wb)
{
	const int total = 9 * cin * n;
	for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x)
	{
		//  forward: k = ((t cin/8 + c) n + nn) 8 + e
		{
			const int e = k & 7, r = k >> 3;
			const int nn = r % n, tc_ = r / n;
			const int t = tc_ / (cin / 8), c = tc_ - t * (cin / 8);
			wf[k] = __float2bfloat16_rn(W[((size_t)nn * 9 + t) * cin + c * 8 + e]);
		}
		//  transposed: k = ((t' n/8 + c') cin + nn') 8 + e'
		{
			const int e = k & 7, r = k >> 3;
			const int nn = r % cin, tc_ = r / cin;
			const int t = tc_ / (n / 8), c = tc_ - t * (n / 8);
			wb[k] = __float2bfloat16_rn(W[((size_t)(c * 8 + e) * 9 + (8 - t)) * cin + nn]);
		}
	}
}

int Blocks(long long work, int bs = 256)
{
	long long g = (work + bs - 1) / bs;
	if(g < 1) g = 1;
	if(g > 148 * 32) g = 148 * 32;
	return (int)g;
}

} // namespace

//==========================================================================
//  Learned
//==========================================================================
Learned::Learned(int device, int nx, int ny, int capacity, unsigned seed, int act)
    : _device(device), _nx(nx), _ny(ny), _n(nx * ny), _act(act ? 1 : 0), _cap(capacity)
{
	if(nx < 8 || ny < 8) throw UsageError("learned: the grid needs at least 8 x 8 points");
	if(capacity < 2) throw UsageError("learned: the sample capacity must be >= 2");
	YZ_CUDA(cudaSetDevice(device));
	_lv[0].W = 8 * ((nx + 7) / 8 + 1);
	_lv[0].H = 8 * ((ny + 7) / 8);
	_lv[0].realW = nx;
	_lv[0].realH = ny;
	for(int l = 1; l < 4; ++l)
	{
		_lv[l].W = _lv[l - 1].W / 2;
		_lv[l].H = _lv[l - 1].H / 2;
		_lv[l].realW = (_lv[l - 1].realW + 1) / 2;
		_lv[l].realH = (_lv[l - 1].realH + 1) / 2;
	}
	const int spec[7][3] = {{16, 16, 0}, {16, 32, 1}, {32, 64, 2}, {64, 64, 3}, {128, 64, 2}, {96, 32, 1}, {48, 16, 0}};
	size_t off = 0, wf = 0;
	for(auto &s : spec)
	{
		ConvLayer L;
		L.cin = s[0]; L.cout = s[1]; L.level = s[2];
		L.wOff = off; off += (size_t)9 * L.cin * L.cout;
		L.bOff = off; off += (size_t)L.cout;
		_conv.push_back(L);
		_wfOff.push_back(wf);
		_wbOff.push_back(wf);
		wf += (size_t)9 * L.cin * L.cout;
	}
	_outW = off; off += 16;
	_outB = off; off += 1;
	_np = off;
	//  He-normal initialisation from a fixed generator; biases 0; the
	//  output layer small
	std::vector<float> h(_np, 0.0f);
	std::mt19937 gen(seed);
	for(const ConvLayer &L : _conv)
	{
		//  He (ReLU) or Glorot-like (linear) scale
		std::normal_distribution<float> nd(0.0f, std::sqrt((_act ? 2.0f : 1.0f) / (9.0f * (float)L.cin)));
		for(size_t k = 0; k < (size_t)9 * L.cin * L.cout; ++k) h[L.wOff + k] = nd(gen);
	}
	{
		std::normal_distribution<float> nd(0.0f, std::sqrt(1.0f / 16.0f));
		for(int c = 0; c < 16; ++c) h[_outW + c] = nd(gen);
	}
	cudaStream_t st = 0;
	_param.upload(h.data(), _np, st);
	_grad.reserve(_np); _m.reserve(_np); _v.reserve(_np);
	YZ_CUDA(cudaMemsetAsync(_m.get(), 0, _np * sizeof(float), st));
	YZ_CUDA(cudaMemsetAsync(_v.get(), 0, _np * sizeof(float), st));
	_wf.reserve(wf); _wb.reserve(wf);
	//  activations
	auto px = [&](int l) { return (size_t)_lv[l].H * _lv[l].W; };
	_F.reserve(px(0) * 16);
	_U0.reserve(px(0) * 48); _P1.reserve(px(1) * 16); _U1.reserve(px(1) * 96); _P2.reserve(px(2) * 32);
	_U2.reserve(px(2) * 128); _P3.reserve(px(3) * 64); _B3.reserve(px(3) * 64); _D2.reserve(px(2) * 64);
	_D1.reserve(px(1) * 32); _D0.reserve(px(0) * 16);
	_T.reserve(px(0));
	_aux.reserve((size_t)2 * _n);
	YZ_CUDA(cudaMemsetAsync(_aux.get(), 0, (size_t)2 * _n * sizeof(float), st));
	_rms.reserve(2); _inv.reserve(2);
	_red.reserve((size_t)RedBlocks(_n));
	_cnt.reserve(4);
	YZ_CUDA(cudaMemsetAsync(_cnt.get(), 0, 4 * sizeof(unsigned int), st));
	_outSum.reserve(4);
	{
		const float one = 1.0f;
		_tsc.upload(&one, 1, st);
	}
	_err.reserve(1);
	YZ_CUDA(cudaMemsetAsync(_err.get(), 0, sizeof(int), st));
	_ring.reserve((size_t)_cap * 4 * _n);
	_valid.reserve((size_t)_cap);
	YZ_CUDA(cudaMemsetAsync(_valid.get(), 0, (size_t)_cap * sizeof(int), st));
	YZ_CUDA(cudaFuncSetAttribute(KConv3x3, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmemMax + 64));
	Pack(st);
	YZ_CUDA(cudaStreamSynchronize(st));
}

Learned::~Learned() { cudaSetDevice(_device); cudaDeviceSynchronize(); }

void Learned::Pack(cudaStream_t st)
{
	for(size_t k = 0; k < _conv.size(); ++k)
	{
		const ConvLayer &L = _conv[k];
		YZ_LAUNCH(KPackW, Blocks((long long)9 * L.cin * L.cout), 256, 0, st, L.cin, L.cout, _param.get() + L.wOff,
		          _wf.get() + _wfOff[k], _wb.get() + _wbOff[k]);
	}
}

void Learned::Conv(const ConvLayer &L, bool transpose, const bf16 *x, bf16 *y, int ldy, int coff, bool relu,
                   cudaStream_t st, const int *halt)
{
	const size_t k = (size_t)(&L - _conv.data());
	ConvArgs a;
	a.x = x; a.y = y;
	a.cin = transpose ? L.cout : L.cin;
	a.n = transpose ? L.cin : L.cout;
	a.w = (transpose ? _wb.get() + _wbOff[k] : _wf.get() + _wfOff[k]);
	a.bias = transpose ? nullptr : _param.get() + L.bOff;
	const Level &lv = _lv[L.level];
	a.H = lv.H; a.W = lv.W; a.realW = lv.realW; a.realH = lv.realH;
	a.ldy = ldy; a.coff = coff; a.relu = relu ? 1 : 0;
	a.tpg = ConvTapsPerGroup(a.cin, a.n);
	a.halt = halt;
	a.err = _err.get();
	const int tiles = (lv.H * lv.W + kTile - 1) / kTile;
	YZ_LAUNCH(KConv3x3, tiles, 128, ConvSmem(a.cin, a.n, a.tpg), st, a);
}

void Learned::ForwardImage(cudaStream_t st, const int *halt)
{
	auto L = [&](int l) { Lv v; v.H = _lv[l].H; v.W = _lv[l].W; v.realH = _lv[l].realH; v.realW = _lv[l].realW; return v; };
	auto px = [&](int l) { return (long long)_lv[l].H * _lv[l].W; };
	const ConvLayer &enc0 = _conv[0], &enc1 = _conv[1], &enc2 = _conv[2], &bott = _conv[3], &dec2 = _conv[4],
	                &dec1 = _conv[5], &dec0 = _conv[6];
	Conv(enc0, false, _F.get(), _U0.get(), 48, 0, _act != 0, st, halt);
	YZ_LAUNCH(KPool, Blocks(px(1) * 2), 256, 0, st, 16, 48, _U0.get(), L(0), _P1.get(), L(1), halt);
	Conv(enc1, false, _P1.get(), _U1.get(), 96, 0, _act != 0, st, halt);
	YZ_LAUNCH(KPool, Blocks(px(2) * 4), 256, 0, st, 32, 96, _U1.get(), L(1), _P2.get(), L(2), halt);
	Conv(enc2, false, _P2.get(), _U2.get(), 128, 0, _act != 0, st, halt);
	YZ_LAUNCH(KPool, Blocks(px(3) * 8), 256, 0, st, 64, 128, _U2.get(), L(2), _P3.get(), L(3), halt);
	Conv(bott, false, _P3.get(), _B3.get(), 64, 0, _act != 0, st, halt);
	YZ_LAUNCH(KUp, Blocks(px(2) * 8), 256, 0, st, 64, _B3.get(), L(3), _U2.get(), 128, 64, L(2), halt);
	Conv(dec2, false, _U2.get(), _D2.get(), 64, 0, _act != 0, st, halt);
	YZ_LAUNCH(KUp, Blocks(px(1) * 8), 256, 0, st, 64, _D2.get(), L(2), _U1.get(), 96, 32, L(1), halt);
	Conv(dec1, false, _U1.get(), _D1.get(), 32, 0, _act != 0, st, halt);
	YZ_LAUNCH(KUp, Blocks(px(0) * 4), 256, 0, st, 32, _D1.get(), L(1), _U0.get(), 48, 16, L(0), halt);
	Conv(dec0, false, _U0.get(), _D0.get(), 16, 0, _act != 0, st, halt);
}

void Learned::WGrad(const ConvLayer &L, const bf16 *x, const bf16 *dy, cudaStream_t st)
{
	const Level &lv = _lv[L.level];
	const int HW = lv.H * lv.W;
	int pb = (HW + 63) / 64;
	pb = ((pb + kWgJ - 1) / kWgJ) * kWgJ;
	if(pb < kWgJ) pb = kWgJ;
	const int nb = (HW + pb - 1) / pb;
	const size_t outs = (size_t)L.cout * L.cin;
	if(outs > (size_t)256 * kWgTiles * 16 || L.cin > 128 || L.cout > 128) throw UsageError("wgrad: layer too wide");
	_part.reserve((size_t)nb * 9 * outs);
	_partB.reserve((size_t)nb * L.cout);
	YZ_LAUNCH(KWGrad, dim3(nb, 9), 256, 0, st, lv.H, lv.W, L.cin, L.cout, pb, x, dy, _part.get(), _partB.get());
	YZ_LAUNCH(KWReduce, Blocks((long long)9 * outs + L.cout), 256, 0, st, nb, L.cin, L.cout, _part.get(), _partB.get(),
	          _grad.get(), L.wOff, L.bOff, _act);
}

void Learned::BackwardImage(cudaStream_t st)
{
	auto L = [&](int l) { Lv v; v.H = _lv[l].H; v.W = _lv[l].W; v.realH = _lv[l].realH; v.realW = _lv[l].realW; return v; };
	auto px = [&](int l) { return (long long)_lv[l].H * _lv[l].W; };
	const ConvLayer &enc0 = _conv[0], &enc1 = _conv[1], &enc2 = _conv[2], &bott = _conv[3], &dec2 = _conv[4],
	                &dec1 = _conv[5], &dec0 = _conv[6];
	_gU0.reserve(px(0) * 48); _gD1.reserve(px(1) * 32); _gE0.reserve(px(0) * 16); _gU1.reserve(px(1) * 96);
	_gD2.reserve(px(2) * 64); _gE1.reserve(px(1) * 32); _gU2.reserve(px(2) * 128); _gB3.reserve(px(3) * 64);
	_gE2.reserve(px(2) * 64); _gP3.reserve(px(3) * 64); _gP2.reserve(px(2) * 32); _gP1.reserve(px(1) * 16);
	//  dec0: gD0 (from the loss) -> gU0; dW
	Conv(dec0, true, _gD0.get(), _gU0.get(), 48, 0, false, st, nullptr);
	WGrad(dec0, _U0.get(), _gD0.get(), st);
	YZ_LAUNCH(KUpBack, Blocks(px(1) * 4), 256, 0, st, 32, _gU0.get(), 48, 16, L(0), _D1.get(), L(1), _gD1.get(), _act);
	//  dec1
	Conv(dec1, true, _gD1.get(), _gU1.get(), 96, 0, false, st, nullptr);
	WGrad(dec1, _U1.get(), _gD1.get(), st);
	YZ_LAUNCH(KUpBack, Blocks(px(2) * 8), 256, 0, st, 64, _gU1.get(), 96, 32, L(1), _D2.get(), L(2), _gD2.get(), _act);
	//  dec2
	Conv(dec2, true, _gD2.get(), _gU2.get(), 128, 0, false, st, nullptr);
	WGrad(dec2, _U2.get(), _gD2.get(), st);
	YZ_LAUNCH(KUpBack, Blocks(px(3) * 8), 256, 0, st, 64, _gU2.get(), 128, 64, L(2), _B3.get(), L(3), _gB3.get(), _act);
	//  bottleneck
	Conv(bott, true, _gB3.get(), _gP3.get(), 64, 0, false, st, nullptr);
	WGrad(bott, _P3.get(), _gB3.get(), st);
	//  enc2
	YZ_LAUNCH(KSkipBack, Blocks(px(2) * 8), 256, 0, st, 64, _gU2.get(), _U2.get(), 128, L(2), _gP3.get(), L(3), _gE2.get(), _act);
	Conv(enc2, true, _gE2.get(), _gP2.get(), 32, 0, false, st, nullptr);
	WGrad(enc2, _P2.get(), _gE2.get(), st);
	//  enc1
	YZ_LAUNCH(KSkipBack, Blocks(px(1) * 4), 256, 0, st, 32, _gU1.get(), _U1.get(), 96, L(1), _gP2.get(), L(2), _gE1.get(), _act);
	Conv(enc1, true, _gE1.get(), _gP1.get(), 16, 0, false, st, nullptr);
	WGrad(enc1, _P1.get(), _gE1.get(), st);
	//  enc0 (no gradient of the input features)
	YZ_LAUNCH(KSkipBack, Blocks(px(0) * 2), 256, 0, st, 16, _gU0.get(), _U0.get(), 48, L(0), _gP1.get(), L(1), _gE0.get(), _act);
	WGrad(enc0, _F.get(), _gE0.get(), st);
}

void Learned::SetAux(const double *dValues, const int *rowptr, const double *h, cudaStream_t st)
{
	YZ_LAUNCH(KAux, Blocks(_n), 256, 0, st, _n, dValues, rowptr, h, _aux.get());
}

void Learned::Apply(const double *r, double *z, cudaStream_t st, const int *halt)
{
	RedScratch rs;
	rs.part = _red.get(); rs.counter = _cnt.get(); rs.maxBlocks = RedBlocks(_n);
	Lv l0; l0.H = _lv[0].H; l0.W = _lv[0].W; l0.realH = _lv[0].realH; l0.realW = _lv[0].realW;
	YZ_LAUNCH(KSumSq, RedBlocks(_n), kRT, 0, st, _n, r, rs, _rms.get(), _inv.get(), halt);
	YZ_LAUNCH(KPackF, Blocks((long long)l0.H * l0.W), 256, 0, st, _n, _nx, l0, r, _inv.get(), _aux.get(), _F.get(), halt);
	ForwardImage(st, halt);
	YZ_LAUNCH(KOut, Blocks(_n), 256, 0, st, _n, _nx, l0, _D0.get(), _param.get() + _outW, _param.get() + _outB,
	          _rms.get(), _tsc.get(), z, halt);
}

void Learned::AddSample(const double *r, const double *z, cudaStream_t st, const int *halt)
{
	const int s = _count % _cap;
	RedScratch rs;
	rs.part = _red.get(); rs.counter = _cnt.get() + 1; rs.maxBlocks = RedBlocks(_n);
	YZ_LAUNCH(KSumSq, RedBlocks(_n), kRT, 0, st, _n, r, rs, _rms.get() + 1, _inv.get() + 1, halt);
	YZ_LAUNCH(KStoreSample, Blocks(_n), 256, 0, st, _n, r, z, _inv.get() + 1, _aux.get(),
	          _ring.get() + (size_t)s * 4 * _n, _valid.get() + s, halt);
	++_count;
}

void Learned::AddSampleHost(const double *r, const double *z, const double *diag, const double *h, cudaStream_t st)
{
	DBuf<double> dr, dz, dd, dh;
	DBuf<int> rp;
	dr.upload(r, (size_t)_n, st);
	dz.upload(z, (size_t)_n, st);
	dd.upload(diag, (size_t)_n, st);
	std::vector<int> ptr((size_t)_n + 1);
	for(int i = 0; i <= _n; ++i) ptr[(size_t)i] = i;
	rp.upload(ptr.data(), ptr.size(), st);
	if(h) dh.upload(h, (size_t)_n, st);
	SetAux(dd.get(), rp.get(), h ? dh.get() : nullptr, st);
	AddSample(dr.get(), dz.get(), st, nullptr);
	YZ_CUDA(cudaStreamSynchronize(st));
}

void Learned::BuildImage(int slot, cudaStream_t st)
{
	Lv l0; l0.H = _lv[0].H; l0.W = _lv[0].W; l0.realH = _lv[0].realH; l0.realW = _lv[0].realW;
	YZ_LAUNCH(KBuildImage, Blocks((long long)l0.H * l0.W), 256, 0, st, _n, _nx, l0,
	          _ring.get() + (size_t)slot * 4 * _n, _tsc.get(), _F.get(), _T.get());
}

void Learned::Check(cudaStream_t st)
{
	int e = 0;
	YZ_CUDA(cudaMemcpyAsync(&e, _err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
	YZ_CUDA(cudaStreamSynchronize(st));
	if(e) throw CudaError("learned: a tensor-core convolution timed out waiting for its MMAs");
}

double Learned::Train(int iters, int batch, float lr, int holdout, double *valErr, cudaStream_t st)
{
	YZ_CUDA(cudaSetDevice(_device));
	const int have = Samples();
	std::vector<int> valid((size_t)have);
	if(have) YZ_CUDA(cudaMemcpyAsync(valid.data(), _valid.get(), (size_t)have * sizeof(int), cudaMemcpyDeviceToHost, st));
	YZ_CUDA(cudaStreamSynchronize(st));
	std::vector<int> slots;
	for(int s = 0; s < have; ++s) if(valid[(size_t)s]) slots.push_back(s);
	if(holdout < 0) holdout = 0;
	if((int)slots.size() <= holdout) throw UsageError("learned: not enough samples to train on");
	std::vector<int> train(slots.begin(), slots.end() - holdout), held(slots.end() - holdout, slots.end());
	Lv l0; l0.H = _lv[0].H; l0.W = _lv[0].W; l0.realH = _lv[0].realH; l0.realW = _lv[0].realW;
	const int lb = (l0.H * l0.W + kRT - 1) / kRT;
	if(!_tscSet)
	{
		//  the targets' scale over the training pairs: the network learns
		//  z / (rms(r) s), whose size is then about 1 whatever the system's
		const int nbz = (_n + kRT - 1) / kRT;
		DBuf<float> part;
		part.reserve((size_t)nbz * train.size());
		for(size_t k = 0; k < train.size(); ++k)
			YZ_LAUNCH(KSlotSq, nbz, kRT, 0, st, _n, _ring.get() + (size_t)train[k] * 4 * _n + _n,
			          part.get() + k * nbz);
		std::vector<float> h((size_t)nbz * train.size());
		part.download(h.data(), h.size(), st);
		YZ_CUDA(cudaStreamSynchronize(st));
		double sum = 0.0;
		for(float v : h) sum += v;
		const double mean = sum / ((double)_n * (double)train.size());
		const float sc = mean > 0 ? (float)std::sqrt(mean) : 1.0f;
		_tsc.upload(&sc, 1, st);
		_tscHost = sc;
		_tscSet = true;
	}
	_gD0.reserve((size_t)l0.H * l0.W * 16);
	_lossPart.reserve((size_t)lb * kLossQ);
	std::mt19937 gen(12345u + (unsigned)_adamT);
	double last = 0.0;
	for(int it = 0; it < iters; ++it)
	{
		YZ_CUDA(cudaMemsetAsync(_grad.get(), 0, _np * sizeof(float), st));
		YZ_CUDA(cudaMemsetAsync(_outSum.get(), 0, sizeof(double), st));
		for(int b = 0; b < batch; ++b)
		{
			const int s = train[(size_t)(gen() % train.size())];
			BuildImage(s, st);
			ForwardImage(st, nullptr);
			YZ_LAUNCH(KLoss, lb, kRT, 0, st, _n, l0, _D0.get(), _T.get(), _param.get() + _outW, _param.get() + _outB,
			          _gD0.get(), _lossPart.get(), _act);
			YZ_LAUNCH(KLossReduce, 1, 32, 0, st, lb, _lossPart.get(), _outSum.get(), _grad.get(), _outW, _outB, _act);
			BackwardImage(st);
		}
		++_adamT;
		const float c1 = 1.0f - std::pow(0.9f, (float)_adamT), c2 = 1.0f - std::pow(0.999f, (float)_adamT);
		YZ_LAUNCH(KAdam, Blocks((long long)_np), 256, 0, st, _np, _param.get(), _grad.get(), _m.get(), _v.get(), lr,
		          1.0f / (float)batch, c1, c2);
		Pack(st);
		if(it == iters - 1)
		{
			double l = 0;
			YZ_CUDA(cudaMemcpyAsync(&l, _outSum.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
			YZ_CUDA(cudaStreamSynchronize(st));
			last = l / batch;
		}
	}
	Check(st);
	_trained = true;
	if(valErr)
	{
		double e = 0.0;
		for(int s : held) e += Validate(s, 1, st);
		*valErr = held.empty() ? -1.0 : e / (double)held.size();
	}
	return last;
}

double Learned::Validate(int first, int count, cudaStream_t st)
{
	Lv l0; l0.H = _lv[0].H; l0.W = _lv[0].W; l0.realH = _lv[0].realH; l0.realW = _lv[0].realW;
	const int lb = (l0.H * l0.W + kRT - 1) / kRT;
	_lossPart.reserve((size_t)lb * kLossQ);
	std::vector<float> part((size_t)2 * lb);
	double sum = 0.0;
	for(int s = first; s < first + count; ++s)
	{
		BuildImage(s % _cap, st);
		ForwardImage(st, nullptr);
		YZ_LAUNCH(KValErr, lb, kRT, 0, st, l0, _D0.get(), _T.get(), _param.get() + _outW, _param.get() + _outB,
		          _lossPart.get());
		YZ_CUDA(cudaMemcpyAsync(part.data(), _lossPart.get(), part.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
		YZ_CUDA(cudaStreamSynchronize(st));
		double e = 0, t = 0;
		for(int b = 0; b < lb; ++b) { e += part[(size_t)2 * b]; t += part[(size_t)2 * b + 1]; }
		sum += t > 0 ? std::sqrt(e / t) : 0.0;
	}
	Check(st);
	return count ? sum / count : 0.0;
}

void Learned::GetParams(float *out, cudaStream_t st)
{
	_param.download(out, _np, st);
	YZ_CUDA(cudaStreamSynchronize(st));
}

bool Learned::GetSample(int k, float *out, cudaStream_t st)
{
	if(k < 0 || k >= Samples()) throw UsageError("unet: no sample in that slot");
	int valid = 0;
	YZ_CUDA(cudaMemcpyAsync(out, _ring.get() + (size_t)k * 4 * _n, (size_t)4 * _n * sizeof(float),
	                        cudaMemcpyDeviceToHost, st));
	YZ_CUDA(cudaMemcpyAsync(&valid, _valid.get() + k, sizeof(int), cudaMemcpyDeviceToHost, st));
	YZ_CUDA(cudaStreamSynchronize(st));
	return valid != 0;
}

void Learned::SetParams(const float *in, cudaStream_t st)
{
	_param.upload(in, _np, st);
	Pack(st);
	YZ_CUDA(cudaStreamSynchronize(st));
}

double Learned::LossGrad(const float *feat3, const float *target, float *grad, cudaStream_t st)
{
	//  the sample into a scratch slot of the ring (the last one), as stored
	//  pairs are: r, z, diag, h maps
	std::vector<float> slot((size_t)4 * _n);
	for(int i = 0; i < _n; ++i)
	{
		slot[(size_t)i] = feat3[i];
		slot[(size_t)_n + i] = target[i];
		slot[(size_t)2 * _n + i] = feat3[_n + i];
		slot[(size_t)3 * _n + i] = feat3[2 * _n + i];
	}
	const int s = _cap - 1;
	YZ_CUDA(cudaMemcpyAsync(_ring.get() + (size_t)s * 4 * _n, slot.data(), slot.size() * sizeof(float),
	                        cudaMemcpyHostToDevice, st));
	Lv l0; l0.H = _lv[0].H; l0.W = _lv[0].W; l0.realH = _lv[0].realH; l0.realW = _lv[0].realW;
	const int lb = (l0.H * l0.W + kRT - 1) / kRT;
	_gD0.reserve((size_t)l0.H * l0.W * 16);
	_lossPart.reserve((size_t)lb * kLossQ);
	YZ_CUDA(cudaMemsetAsync(_grad.get(), 0, _np * sizeof(float), st));
	YZ_CUDA(cudaMemsetAsync(_outSum.get(), 0, sizeof(double), st));
	BuildImage(s, st);
	ForwardImage(st, nullptr);
	YZ_LAUNCH(KLoss, lb, kRT, 0, st, _n, l0, _D0.get(), _T.get(), _param.get() + _outW, _param.get() + _outB,
	          _gD0.get(), _lossPart.get(), _act);
	YZ_LAUNCH(KLossReduce, 1, 32, 0, st, lb, _lossPart.get(), _outSum.get(), _grad.get(), _outW, _outB, _act);
	BackwardImage(st);
	double l = 0;
	YZ_CUDA(cudaMemcpyAsync(&l, _outSum.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
	_grad.download(grad, _np, st);
	YZ_CUDA(cudaStreamSynchronize(st));
	Check(st);
	return l;
}

void Learned::Forward(const float *feat3, float *out, cudaStream_t st)
{
	std::vector<float> slot((size_t)4 * _n, 0.0f);
	for(int i = 0; i < _n; ++i)
	{
		slot[(size_t)i] = feat3[i];
		slot[(size_t)2 * _n + i] = feat3[_n + i];
		slot[(size_t)3 * _n + i] = feat3[2 * _n + i];
	}
	const int s = _cap - 1;
	YZ_CUDA(cudaMemcpyAsync(_ring.get() + (size_t)s * 4 * _n, slot.data(), slot.size() * sizeof(float),
	                        cudaMemcpyHostToDevice, st));
	Lv l0; l0.H = _lv[0].H; l0.W = _lv[0].W; l0.realH = _lv[0].realH; l0.realW = _lv[0].realW;
	BuildImage(s, st);
	ForwardImage(st, nullptr);
	DBuf<float> o;
	o.reserve((size_t)_n);
	YZ_LAUNCH(KOutMap, Blocks(_n), 256, 0, st, _n, _nx, l0, _D0.get(), _param.get() + _outW, _param.get() + _outB,
	          o.get());
	o.download(out, (size_t)_n, st);
	YZ_CUDA(cudaStreamSynchronize(st));
	for(int i = 0; i < _n; ++i) out[i] *= _tscHost;
	Check(st);
}

//==========================================================================
//  one convolution on host arrays (the tensor-core kernel's parity test)
//==========================================================================
void Conv3x3Host(int H, int W, int cin, int n, int realW, int realH, int relu, const float *x, const float *w,
                 const float *bias, float *y)
{
	if(cin % 16 || n % 16 || cin > 128 || n > 256 || cin <= 0 || n <= 0) throw UsageError("conv3x3: cin and n must be multiples of 16 (cin <= 128, n <= 256)");
	if(H <= 0 || W <= 0 || realW > W || realH > H) throw UsageError("conv3x3: bad image size");
	cudaStream_t st = 0;
	const size_t HW = (size_t)H * W;
	std::vector<bf16> hx(HW * cin);
	for(size_t k = 0; k < hx.size(); ++k) hx[k] = __float2bfloat16_rn(x[k]);
	DBuf<bf16> dx, dy, dwf, dwb;
	DBuf<float> dW, db;
	DBuf<int> err;
	dx.upload(hx.data(), hx.size(), st);
	dy.reserve(HW * n);
	dW.upload(w, (size_t)9 * cin * n, st);
	if(bias) db.upload(bias, (size_t)n, st);
	dwf.reserve((size_t)9 * cin * n);
	dwb.reserve((size_t)9 * cin * n);
	err.reserve(1);
	YZ_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
	YZ_CUDA(cudaFuncSetAttribute(KConv3x3, cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmemMax + 64));
	YZ_LAUNCH(KPackW, Blocks((long long)9 * cin * n), 256, 0, st, cin, n, dW.get(), dwf.get(), dwb.get());
	ConvArgs a;
	a.x = dx.get(); a.y = dy.get(); a.w = dwf.get(); a.bias = bias ? db.get() : nullptr;
	a.H = H; a.W = W; a.cin = cin; a.n = n; a.ldy = n; a.coff = 0; a.realW = realW; a.realH = realH;
	a.relu = relu; a.tpg = ConvTapsPerGroup(cin, n); a.halt = nullptr; a.err = err.get();
	YZ_LAUNCH(KConv3x3, (int)((HW + kTile - 1) / kTile), 128, ConvSmem(cin, n, a.tpg), st, a);
	std::vector<bf16> hy(HW * n);
	dy.download(hy.data(), hy.size(), st);
	int e = 0;
	YZ_CUDA(cudaMemcpyAsync(&e, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
	YZ_CUDA(cudaStreamSynchronize(st));
	if(e) throw CudaError("conv3x3: the tensor-core convolution timed out waiting for its MMAs");
	for(size_t k = 0; k < hy.size(); ++k) y[k] = __bfloat162float(hy[k]);
}

} // namespace yz
