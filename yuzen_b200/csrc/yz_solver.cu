// yz_solver.cu -- the linear solve of the implicit step on the device: the
// drop-in for ILinearSolverBackend::Solve (LinearSolverBackend.h:74-88).
//
// The flow of one solve follows AmgclBackend::Solve
// (LinearSolverBackend.cpp:539-728): row scaling into the sorted mirror,
// SPAI0 tried first on a concentration solve (TryBackoff, :262-270), then
// BiCGStab preconditioned by SA-AMG(SPAI0) rebuilt for every solve (ILU) or
// by damped Jacobi (None, Jacobi), coarse_enough 500 above 3000 rows (:660-675),
// a breakdown answered by the residual check of :681-713.
#include "yz_amg_kernels.cuh"
#include "yz_coarse.cuh"
#include "yz_learned.h"
#include "yz_solver_impl.h"
#include "yz_prof.h"

#include <map>
#include <mutex>
#include <type_traits>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace yz {

//==========================================================================
//  Krylov kernels: element-wise updates fused with the dot products they
//  feed, all on the chunk mapping of the reduction tree (block b, thread t:
//  elements b*4096 + k*256 + t).  Scalars live in device memory (Scal).
//==========================================================================
#define YZ_CHUNK_LOOP(i)                                                          \
	for(int kk_ = 0, i = blockIdx.x * kRChunk + threadIdx.x; kk_ < kRK; ++kk_, i += kRT)

//  r = b - A x;  bb = b.b, rr = r.r, rho0 = r.r (rh = r)
template<class V>
__global__ void __launch_bounds__(kRT, 8) KBInit(int n, const int *__restrict__ ptr, const int *__restrict__ sellOff, Sten sn, const int *__restrict__ col,
                       const V *__restrict__ val, const double *__restrict__ b,
                       const double *__restrict__ x, double *__restrict__ r, double *__restrict__ rh,
                       RedScratch rs, Scal *sc)
{
	__shared__ double sh[2 * kRT];
	double a[2] = {0.0, 0.0};
	YZ_CHUNK_LOOP(i)
	{
		if(i >= n) break;
		int st, len, sd;
		RowRange(ptr, sellOff, i, st, len, sd);
		const double s = RowSumSten(sn, i, st, len, sd, col, val, [&](int c) { return x[c]; });
		const double ri = b[i] - s;
		r[i] = ri; rh[i] = ri;
		a[0] = a[0] + b[i] * b[i];
		a[1] = a[1] + ri * ri;
	}
	double tot[2];
	if(GridFold<2>(a, sh, rs, tot) && threadIdx.x == 0)
	{
		sc->normb = sqrt(tot[0]);
		sc->res = sqrt(tot[1]);
		sc->rho = tot[1];
	}
}

//  The top of an iteration (the oracle's `while(it < maxIter)` and its
//  breakdown test), then p = r (first pass) or p = r + beta (p - omega v)
__global__ void KPUpdate(int n, const double *__restrict__ r, const double *__restrict__ v,
                         double *__restrict__ p, Scal *sc)
{
	PdlEntry();
	if(sc->state != kRun) return;
	const bool lead = (blockIdx.x == 0 && threadIdx.x == 0);
	if(sc->it >= sc->maxIter) { if(lead) sc->state = kCap; return; }
	if(sc->rho == 0.0) { if(lead) sc->state = kBreak; return; }
	const int first = (sc->it == 0);
	if(first)
	{
		for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = r[i];
		return;
	}
	const double omega = sc->omega;
	const double beta = (sc->rho / sc->rhoPrev) * (sc->alpha / omega);
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

//  v = A ph; alpha = rho / (rh . v)
template<class V>
__global__ void __launch_bounds__(kRT, 8) KSpmvAlpha(int n, const int *__restrict__ ptr, const int *__restrict__ sellOff, Sten sn,
                           const int *__restrict__ col, const V *__restrict__ val, const double *__restrict__ ph,
                           const double *__restrict__ rh, double *__restrict__ v, RedScratch rs, Scal *sc)
{
	PdlEntry();
	if(sc->state != kRun) return;
	__shared__ double sh[kRT];
	double a[1] = {0.0};
	YZ_CHUNK_LOOP(i)
	{
		if(i >= n) break;
		int st, len, sd;
		RowRange(ptr, sellOff, i, st, len, sd);
		const double s = RowSumSten(sn, i, st, len, sd, col, val, [&](int c) { return ph[c]; });
		v[i] = s;
		a[0] = a[0] + rh[i] * s;
	}
	double tot[1];
	if(GridFold<1>(a, sh, rs, tot) && threadIdx.x == 0) sc->alpha = sc->rho / tot[0];
}

//  s = r - alpha v; res = |s|
__global__ void KSUpdate(int n, const double *__restrict__ r, const double *__restrict__ v,
                         double *__restrict__ s, RedScratch rs, Scal *sc)
{
	PdlEntry();
	if(sc->state != kRun) return;
	__shared__ double sh[kRT];
	const double alpha = sc->alpha;
	double a[1] = {0.0};
	YZ_CHUNK_LOOP(i)
	{
		if(i >= n) break;
		const double si = r[i] - alpha * v[i];
		s[i] = si;
		a[0] = a[0] + si * si;
	}
	double tot[1];
	if(GridFold<1>(a, sh, rs, tot) && threadIdx.x == 0)
	{
		const double res = sqrt(tot[0]);
		sc->res = res;
		//  converged at the half step: x takes alpha ph (in KXRUpdate) and the
		//  iteration counts
		if(res <= sc->eps) { sc->state = kConvHalf; sc->it += 1; }
	}
}

//  t = A sh; omega = (t . s) / (t . t)
template<class V>
__global__ void __launch_bounds__(kRT, 8) KSpmvOmega(int n, const int *__restrict__ ptr, const int *__restrict__ sellOff, Sten sn,
                           const int *__restrict__ col, const V *__restrict__ val, const double *__restrict__ sh_,
                           const double *__restrict__ s, double *__restrict__ t, RedScratch rs, Scal *sc)
{
	PdlEntry();
	if(sc->state != kRun) return;
	__shared__ double sh[2 * kRT];
	double a[2] = {0.0, 0.0};
	YZ_CHUNK_LOOP(i)
	{
		if(i >= n) break;
		int st, len, sd;
		RowRange(ptr, sellOff, i, st, len, sd);
		const double u = RowSumSten(sn, i, st, len, sd, col, val, [&](int c) { return sh_[c]; });
		t[i] = u;
		a[0] = a[0] + u * u;
		a[1] = a[1] + u * s[i];
	}
	double tot[2];
	if(GridFold<2>(a, sh, rs, tot) && threadIdx.x == 0) sc->omega = tot[1] / tot[0];
}

//  x = (x + alpha ph) + omega sh; r = s - omega t; res = |r|; next rho = rh . r.
//  After a half-step exit (KSUpdate set kConvHalf, the rest of the iteration
//  did nothing): x = x + alpha ph instead; the iteration's end turns the
//  state into kConv, so that no later kernel repeats it.
__global__ void KXRUpdate(int n, const double *__restrict__ ph, const double *__restrict__ shat,
                          const double *__restrict__ s, const double *__restrict__ t,
                          const double *__restrict__ rh, double *__restrict__ x, double *__restrict__ r,
                          RedScratch rs, Scal *sc)
{
	PdlEntry();
	const int state = sc->state;
	if(state == kConvHalf)
	{
		const double alpha = sc->alpha;
		YZ_CHUNK_LOOP(i)
		{
			if(i >= n) break;
			x[i] = x[i] + alpha * ph[i];
		}
		return;
	}
	if(state != kRun) return;
	__shared__ double sh[2 * kRT];
	const double alpha = sc->alpha, omega = sc->omega;
	double a[2] = {0.0, 0.0};
	YZ_CHUNK_LOOP(i)
	{
		if(i >= n) break;
		x[i] = (x[i] + alpha * ph[i]) + omega * shat[i];
		const double ri = s[i] - omega * t[i];
		r[i] = ri;
		a[0] = a[0] + ri * ri;
		a[1] = a[1] + rh[i] * ri;
	}
	double tot[2];
	if(GridFold<2>(a, sh, rs, tot) && threadIdx.x == 0)
	{
		const double res = sqrt(tot[0]);
		sc->res = res;
		sc->rhoPrev = sc->rho;
		sc->rho = tot[1];
		sc->it += 1;
		if(res <= sc->eps) sc->state = kConv;
		else if(!(res == res)) sc->state = kNaN;
	}
}

//  the start of the iterations: the tolerance, the cap, the counters
__global__ void KCtlInit(Scal *sc, double eps, int maxIter)
{
	sc->eps = eps; sc->maxIter = maxIter; sc->it = 0; sc->state = kRun; sc->bodies = 0;
}

//  The start of a run from KBInit's norms, on the device (the oracle's tests
//  before its loop): |b| < 2 eps_machine gives x = 0 and no iteration; else
//  eps = tol |b|, and the loop runs while the start residual is above it and
//  an iteration is allowed
__global__ void KCtlStart(Scal *sc, double tol, int maxIter)
{
	sc->maxIter = maxIter; sc->it = 0; sc->bodies = 0;
	const double normB = sc->normb;
	if(normB < 2.0 * 2.220446049250313e-16) { sc->state = kTiny; return; }
	const double eps = tol * normB;
	sc->eps = eps;
	sc->state = (sc->res > eps && maxIter > 0) ? kRun : kSkip;
}

__global__ void KZeroIfTiny(int n, const Scal *sc, double *__restrict__ x)
{
	if(sc->state != kTiny) return;
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = 0.0;
}

//  The end of an iteration: a half-step exit, whose x update KXRUpdate has just
//  made, becomes a plain exit, so that an iteration queued after it makes
//  no second one; then the loop's condition (another iteration while the
//  run goes on)
__global__ void KLoopCond(cudaGraphConditionalHandle h, Scal *sc)
{
	sc->bodies += 1;
	if(sc->state == kConvHalf) sc->state = kConv;
	cudaGraphSetConditional(h, sc->state == kRun ? 1u : 0u);
}

//  the same where the iterations are queued one by one
__global__ void KLoopCount(Scal *sc)
{
	sc->bodies += 1;
	if(sc->state == kConvHalf) sc->state = kConv;
}

__global__ void KFill(int n, double v, double *__restrict__ x)
{
	for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

//  the deterministic dot product on its own (for the parity tests)
__global__ void KDot(int n, const double *__restrict__ x, const double *__restrict__ y, RedScratch rs, double *out)
{
	__shared__ double sh[kRT];
	double a[1] = {0.0};
	YZ_CHUNK_LOOP(i)
	{
		if(i >= n) break;
		a[0] = a[0] + x[i] * y[i];
	}
	double tot[1];
	if(GridFold<1>(a, sh, rs, tot) && threadIdx.x == 0) *out = tot[0];
}

#undef YZ_CHUNK_LOOP

//==========================================================================
//  Fault injection: the switch of the reference's amgcl backend
//  (LinearSolverBackend.cpp:630-645).  YUZEN_FAULT_AMGCL=k:m (read at the
//  first solve) or FaultInject(k, m) makes m solves of the process, from the
//  k-th of those that reach the SA-AMG / Jacobi path on, break down before
//  they iterate -- the reference's "Zero rho in BiCGStab" -- so that the
//  caller sees the breakdown return (2) and the step its cut-and-retry.
//==========================================================================
namespace {
struct FaultState
{
	long at = 0, count = 0, solves = 0;
	bool read = false;
};
std::mutex g_faultMutex;
FaultState g_fault;

bool FaultNow()
{
	std::lock_guard<std::mutex> lk(g_faultMutex);
	if(!g_fault.read)
	{
		g_fault.read = true;
		if(const char *e = std::getenv("YUZEN_FAULT_AMGCL"))
		{
			char *end = nullptr;
			g_fault.at = std::strtol(e, &end, 10);
			g_fault.count = (end && *end == ':') ? std::strtol(end + 1, nullptr, 10) : 1;
		}
	}
	return g_fault.at > 0 && ++g_fault.solves >= g_fault.at && g_fault.solves < g_fault.at + g_fault.count;
}
} // namespace

void FaultInject(long at, long count)
{
	std::lock_guard<std::mutex> lk(g_faultMutex);
	g_fault.read = true;
	g_fault.at = at;
	g_fault.count = count;
	g_fault.solves = 0;
}

//==========================================================================
//  Solver
//==========================================================================
static const int kB = 256;

Solver::Solver(int device, cudaStream_t stream) : _device(device)
{
	YZ_CUDA(cudaSetDevice(device));
	if(stream) { _st = stream; _ownStream = false; }
	else YZ_CUDA(cudaStreamCreateWithFlags(&_st, cudaStreamNonBlocking));
	YZ_CUDA(cudaEventCreate(&_ev0)); YZ_CUDA(cudaEventCreate(&_ev1)); YZ_CUDA(cudaEventCreate(&_ev2));
	YZ_CUDA(cudaMallocHost(&_hsc, sizeof(Scal)));
	YZ_CUDA(cudaMallocHost(&_hint, 4 * sizeof(int)));
	YZ_CUDA(cudaMallocHost(&_hring, 2 * sizeof(Scal)));
	YZ_CUDA(cudaEventCreateWithFlags(&_evRing[0], cudaEventDisableTiming));
	YZ_CUDA(cudaEventCreateWithFlags(&_evRing[1], cudaEventDisableTiming));
	_sc.reserve(1);
	_counters.reserve(16);
	YZ_CUDA(cudaMemsetAsync(_counters.get(), 0, 16 * sizeof(unsigned), _st));
	_flags.reserve(8);
	_coarseBar.reserve(2);
	_coarseErr.reserve(1);
	YZ_CUDA(cudaMemsetAsync(_coarseBar.get(), 0, 2 * sizeof(unsigned), _st));
	YZ_CUDA(cudaMemsetAsync(_coarseErr.get(), 0, sizeof(int), _st));
}

Solver::~Solver()
{
	cudaSetDevice(_device);
	cudaStreamSynchronize(_st);
	if(_hsc) cudaFreeHost(_hsc);
	if(_hint) cudaFreeHost(_hint);
	if(_hring) cudaFreeHost(_hring);
	cudaEventDestroy(_evRing[0]); cudaEventDestroy(_evRing[1]);
	cudaEventDestroy(_ev0); cudaEventDestroy(_ev1); cudaEventDestroy(_ev2);
	FreeLoopGraph(_loop[0]); FreeLoopGraph(_loop[1]); FreeLoopGraph(_loop[2]);
	if(_ownStream) cudaStreamDestroy(_st);
}

RedScratch Solver::Red(int site)
{
	RedScratch r;
	r.part = _part.get();
	r.counter = _counters.get() + site;
	r.maxBlocks = _partBlocks;
	return r;
}

void Solver::SetPattern(int n, int nnz, const int *rowptr, const int *scol, const int *ssrc)
{
	if(n <= 0 || nnz < n) throw UsageError("set_pattern: need n > 0 and nnz >= n");
	YZ_CUDA(cudaSetDevice(_device));
	++_epoch;
	_n = n; _nnz = nnz;
	_hptr.assign(rowptr, rowptr + n + 1);
	if(_hptr[0] != 0 || _hptr[(size_t)n] != nnz) throw UsageError("set_pattern: rowptr[0] must be 0 and rowptr[n] == nnz");
	for(int i = 0; i < n; ++i) if(_hptr[(size_t)i + 1] <= _hptr[(size_t)i]) throw UsageError("set_pattern: every row needs its diagonal");
	for(int k = 0; k < nnz; ++k)
		if(scol[k] < 0 || scol[k] >= n || ssrc[k] < 0 || ssrc[k] >= nnz) throw UsageError("set_pattern: index out of range");
	_hcol.assign(scol, scol + nnz);
	//  the SELL-32 copy of the finest level: slice offsets and columns (the
	//  padding of a short row is never read)
	{
		const int S = (n + 31) / 32;
		std::vector<int> off((size_t)S + 1, 0);
		for(int sl = 0; sl < S; ++sl)
		{
			int w = 0;
			for(int r = 32 * sl; r < std::min(n, 32 * sl + 32); ++r) w = std::max(w, _hptr[(size_t)r + 1] - _hptr[(size_t)r]);
			off[(size_t)sl + 1] = off[(size_t)sl] + 32 * w;
		}
		std::vector<int> scl((size_t)off[(size_t)S], 0);
		for(int i = 0; i < n; ++i)
		{
			const int base = off[(size_t)(i >> 5)] + (i & 31);
			for(int k = _hptr[(size_t)i], e = 0; k < _hptr[(size_t)i + 1]; ++k, ++e) scl[(size_t)base + 32 * e] = scol[k];
			for(int e = _hptr[(size_t)i + 1] - _hptr[(size_t)i]; 32 * e + base < off[(size_t)(i >> 5) + 1]; ++e)
				scl[(size_t)base + 32 * e] = i;
		}
		_sellOff.upload(off.data(), off.size(), _st);
		_sellCol.upload(scl.data(), scl.size(), _st);
		_sellVal.reserve(scl.size());
		YZ_CUDA(cudaMemsetAsync(_sellVal.get(), 0, scl.size() * sizeof(double), _st));
		_sellSize = scl.size();
		//  the stencil: the most common column set relative to the row
		//  (up to 16 entries), and the slices all of whose rows have it
		std::map<std::vector<int>, int> seen;
		std::vector<int> rel;
		for(int i = 0; i < n; ++i)
		{
			const int a = _hptr[(size_t)i], b = _hptr[(size_t)i + 1];
			if(b - a > 16) continue;
			rel.clear();
			for(int k = a; k < b; ++k) rel.push_back(scol[k] - i);
			++seen[rel];
		}
		std::vector<int> best;
		int bestCount = 0;
		for(auto &kv : seen) if(kv.second > bestCount) { best = kv.first; bestCount = kv.second; }
		std::vector<unsigned char> flag((size_t)S, 0);
		int flagged = 0;
		for(int sl = 0; sl < S && !best.empty(); ++sl)
		{
			bool all = true;
			for(int i = 32 * sl; i < std::min(n, 32 * sl + 32) && all; ++i)
			{
				const int a = _hptr[(size_t)i], b = _hptr[(size_t)i + 1];
				if(b - a != (int)best.size()) { all = false; break; }
				for(int k = a; k < b; ++k) if(scol[k] - i != best[(size_t)(k - a)]) { all = false; break; }
			}
			flag[(size_t)sl] = all ? 1 : 0;
			flagged += all ? 1 : 0;
		}
		_sten = Sten();
		if(flagged > 0)
		{
			_stenSlice.upload(flag.data(), flag.size(), _st);
			_sten.slice = _stenSlice.get();
			_sten.len = (int)best.size();
			for(size_t k = 0; k < best.size(); ++k) _sten.off[k] = best[k];
		}
	}
	_levels.clear();
	_levels.emplace_back(new Level());
	_nlev = 1;
	Level &L0 = *_levels[0];
	L0.n = n; L0.nnz = nnz;
	L0.ptr.upload(rowptr, (size_t)n + 1, _st);
	L0.col.upload(scol, (size_t)nnz, _st);
	L0.val.reserve((size_t)nnz);
	_ssrc.upload(ssrc, (size_t)nnz, _st);
	_values.reserve((size_t)nnz);
	_rhs.reserve((size_t)n);
	for(DBuf<double> *v : {&_b, &_x, &_x0, &_r, &_rh, &_p, &_v, &_s, &_ph, &_sh, &_t, &_m})
		v->reserve((size_t)n);
	_partBlocks = RedBlocks(n);
	_part.reserve((size_t)2 * _partBlocks);
	//  set-up scratch, sized by the finest level
	_dia.reserve((size_t)n); _strong.reserve((size_t)nnz); _icnt.reserve((size_t)n + 1);
	_iptr.reserve((size_t)n + 1); _icol.reserve((size_t)nnz); _ifill.reserve((size_t)n + 1);
	_state.reserve((size_t)n); _iso.reserve((size_t)n);
	_T0.reserve((size_t)n); _T1.reserve((size_t)n);
	_flag.reserve((size_t)n + 1); _rootId.reserve((size_t)n + 1); _first.reserve((size_t)n);
	_cnt.reserve((size_t)n + 1);
	_scan.reserve(ScanScratchSize(n + 1) + 4);
	_haveH = false;
	YZ_CUDA(cudaStreamSynchronize(_st));
}

int Solver::ReadInt(const int *d)
{
	int h = 0;
	YZ_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	return h;
}

void Solver::ReadScal()
{
	YZ_CUDA(cudaMemcpyAsync(_hsc, _sc.get(), sizeof(Scal), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
}

//  rows -> scanned row pointer; returns the total
int Solver::ScanCounts(const int *cnt, int *out, int n, const int *flag, int *flagOut)
{
	ScanExclusive(cnt, out, n, _scan.get(), _st);
	if(!flag) return ReadInt(out + n);
	//  the total and a flag in one round trip
	YZ_CUDA(cudaMemcpyAsync(_hint, out + n, sizeof(int), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaMemcpyAsync(_hint + 1, flag, sizeof(int), cudaMemcpyDeviceToHost, _st));
	YZ_CUDA(cudaStreamSynchronize(_st));
	*flagOut = _hint[1];
	return _hint[0];
}

//  C = X Y: one warp per row with room for 64 distinct columns (KGemmWarp),
//  each row computed once into a staging slot and moved to its place after
//  the counts are scanned; the thread-per-row kernels with kRowCap where a
//  row needs more; returns nnz(C)
int Solver::Gemm(int nx, const int *xptr, const int *xcol, const double *xval, const int *yptr, const int *ycol,
                 const double *yval, DBuf<int> &cptr, DBuf<int> &ccol, DBuf<double> &cval)
{
	int *overflow = _flags.get() + 1;
	const int g = GridFor(nx, 128);
	const int gw = GridFor((long long)nx * 32, 256, 148 * 64);
	YZ_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int), _st));
	//  one pass: every row into a staging slot of 64, with its count
	_gtCol.reserve((size_t)nx * 64); _gtVal.reserve((size_t)nx * 64);
	YZ_LAUNCH((KGemmWarp<64, true>), gw, 256, 0, _st, nx, xptr, xcol, xval, yptr, ycol, yval, _cnt.get(), nullptr,
	          _gtCol.get(), _gtVal.get(), overflow);
	cptr.reserve((size_t)nx + 1);
	int ovf = 0;
	int nnz = ScanCounts(_cnt.get(), cptr.get(), nx, overflow, &ovf);
	const bool wide = ovf != 0;
	if(wide)
	{
		YZ_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int), _st));
		YZ_LAUNCH(KGemmCount<kRowCap>, g, 128, 0, _st, nx, xptr, xcol, yptr, ycol, _cnt.get(), overflow);
		nnz = ScanCounts(_cnt.get(), cptr.get(), nx);
		if(ReadInt(overflow)) throw CudaError("AMG set-up: a row of a product gathered more than 256 distinct columns");
	}
	ccol.reserve((size_t)nnz); cval.reserve((size_t)nnz);
	if(wide) YZ_LAUNCH(KGemmFill<kRowCap>, g, 128, 0, _st, nx, xptr, xcol, xval, yptr, ycol, yval, cptr.get(), ccol.get(), cval.get());
	else YZ_LAUNCH(KGemmCompact<64>, GridFor((long long)nx * 64, 256, 148 * 64), 256, 0, _st, nx, cptr.get(),
	               _gtCol.get(), _gtVal.get(), ccol.get(), cval.get());
	return nnz;
}

//  The dense inverse of the direct level (KGjPanel / KGjUpdate): panels of B
//  columns, B as large as fits the panel block's shared memory (32 below
//  ~770 rows)
void Solver::DirectInverse(Level &L)
{
	const int n = L.n;
	if(n > 3000) throw UsageError("AMG set-up: the direct level has more than 3000 rows");
	const size_t w = 2 * (size_t)n;
	_gj[0].reserve((size_t)n * w);
	_gj[1].reserve((size_t)32 * n);
	_gjPiv.reserve(32);
	_gjRow.reserve(32);
	double *Mc = _gj[0].get(), *F = _gj[1].get();
	YZ_CUDA(cudaMemsetAsync(Mc, 0, (size_t)n * w * sizeof(double), _st));
	YZ_LAUNCH(KGjInit, GridFor(n, kB), kB, 0, _st, n, L.ptr.get(), L.col.get(), L.val.get(), Mc);
	const size_t maxSmem = 200 * 1024;
	int B = (int)std::min<size_t>(32, (maxSmem - 512 * 12) / ((size_t)n * sizeof(double)));
	if(B < 1) B = 1;
	static bool attrSet = false;
	if(!attrSet)
	{
		YZ_CUDA(cudaFuncSetAttribute(KGjPanel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxSmem));
		YZ_CUDA(cudaFuncSetAttribute(KGjUpdate, cudaFuncAttributeMaxDynamicSharedMemorySize, 3000 * 8));
		attrSet = true;
	}
	for(int k0 = 0; k0 < n; k0 += B)
	{
		const int b = std::min(B, n - k0);
		const size_t smem = (size_t)b * n * sizeof(double) + 512 * (sizeof(double) + sizeof(int));
		YZ_LAUNCH(KGjPanel, 1, 512, smem, _st, n, k0, b, Mc, F, _gjRow.get(), _gjPiv.get());
		const int jStart = k0 + b, cols = (int)w - jStart;
		if(cols > 0)
			YZ_LAUNCH(KGjUpdate, cols, 128, (size_t)n * sizeof(double), _st, n, k0, b, jStart, Mc, F, _gjRow.get(),
			          _gjPiv.get());
	}
	L.inv.reserve((size_t)n * n);
	YZ_LAUNCH(KGjExtract, GridFor((long long)n * n, kB), kB, 0, _st, n, Mc, L.inv.get());
}

//--------------------------------------------------------------------------
//  the hierarchy
//--------------------------------------------------------------------------
void Solver::BuildHierarchy(int coarseEnough)
{
	//  the levels of the last set-up are reused with their buffers (which
	//  only grow): no device allocation or free once the sizes have settled
	++_epochH;
	++_rebuilds;
	_nlev = 1;
	double eps = 0.08;
	for(size_t l = 0;; ++l)
	{
		Level &L = *_levels[l];
		const int n = L.n, nnz = L.nnz;
		const int g = GridFor(n, kB), gz = GridFor(nnz, kB);
		L.M.reserve((size_t)n); L.f.reserve((size_t)n); L.x.reserve((size_t)n);
		L.t.reserve((size_t)n); L.xt.reserve((size_t)n); L.agg.reserve((size_t)n);
		L.direct = false; L.nc = 0; L.pnnz = 0;
		if(n <= coarseEnough)
		{
			L.direct = true;
			DirectInverse(L);
			break;
		}
		//  strength
		YZ_LAUNCH(KDiag, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), L.val.get(), _dia.get());
		YZ_CUDA(cudaMemsetAsync(_icnt.get(), 0, ((size_t)n + 1) * sizeof(int), _st));
		YZ_LAUNCH(KStrength, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), L.val.get(), _dia.get(), eps * eps,
		          _strong.get(), _icnt.get());
		eps *= 0.5;
		ScanExclusive(_icnt.get(), _iptr.get(), n, _scan.get(), _st);
		YZ_CUDA(cudaMemcpyAsync(_ifill.get(), _iptr.get(), (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, _st));
		YZ_LAUNCH(KFillIn, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), _ifill.get(), _icol.get());
		//  MIS-2 (at most 64 rounds, as the oracle)
		YZ_LAUNCH(KMisInit, g, kB, 0, _st, n, L.ptr.get(), _strong.get(), _iptr.get(), _state.get(), _iso.get());
		int *undec = _flags.get() + 4;		// two counters, by round parity
		YZ_CUDA(cudaMemsetAsync(undec, 0, 2 * sizeof(int), _st));
		YZ_LAUNCH(KMisPack, g, kB, 0, _st, n, _state.get(), _T0.get(), undec);
		for(int round = 0; round < 64; ++round)
		{
			int *u = undec + (round & 1), *un = undec + ((round + 1) & 1);
			YZ_LAUNCH(KMisMax, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), _iptr.get(), _icol.get(),
			          _T0.get(), _T1.get(), u, un);
			YZ_LAUNCH(KMisMax, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), _iptr.get(), _icol.get(),
			          _T1.get(), _T0.get(), u, nullptr);
			YZ_LAUNCH(KMisUpdate, g, kB, 0, _st, n, _state.get(), _T0.get(), u, un);
			if((round & 3) == 3 && ReadInt(un) == 0) break;
		}
		//  aggregates
		YZ_LAUNCH(KRootFlags, g, kB, 0, _st, n, _state.get(), _flag.get());
		const int nc = ScanCounts(_flag.get(), _rootId.get(), n);
		YZ_LAUNCH(KAssignFirst, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), _iptr.get(), _icol.get(),
		          _state.get(), _iso.get(), _rootId.get(), _first.get());
		YZ_LAUNCH(KAssignSecond, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), _iptr.get(), _icol.get(),
		          _iso.get(), _first.get(), L.agg.get());
		YZ_LAUNCH(KSpai0, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), L.val.get(), L.M.get());
		L.nc = nc;
		if(nc == 0) break;		// nothing to coarsen: this level is smoothed only
		//  P
		int *overflow = _flags.get() + 1;
		YZ_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int), _st));
		YZ_LAUNCH(KPCount<32>, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), L.agg.get(), _cnt.get(),
		          overflow);
		L.pptr.reserve((size_t)n + 1);
		int ovfP = 0;
		L.pnnz = ScanCounts(_cnt.get(), L.pptr.get(), n, overflow, &ovfP);
		const bool wideP = ovfP != 0;
		if(wideP)
		{
			YZ_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int), _st));
			YZ_LAUNCH(KPCount<kRowCap>, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), _strong.get(), L.agg.get(),
			          _cnt.get(), overflow);
			L.pnnz = ScanCounts(_cnt.get(), L.pptr.get(), n);
			if(ReadInt(overflow)) throw CudaError("AMG set-up: a row of P gathered more than 256 distinct aggregates");
		}
		L.pcol.reserve((size_t)L.pnnz); L.pval.reserve((size_t)L.pnnz);
		if(wideP)
			YZ_LAUNCH(KPFill<kRowCap>, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), L.val.get(), _strong.get(), L.agg.get(),
			          L.pptr.get(), L.pcol.get(), L.pval.get());
		else
			YZ_LAUNCH(KPFill<32>, g, kB, 0, _st, n, L.ptr.get(), L.col.get(), L.val.get(), _strong.get(), L.agg.get(),
			          L.pptr.get(), L.pcol.get(), L.pval.get());
		//  R = P^T
		L.rptr.reserve((size_t)nc + 1); L.rcol.reserve((size_t)L.pnnz); L.rval.reserve((size_t)L.pnnz);
		YZ_CUDA(cudaMemsetAsync(_cnt.get(), 0, ((size_t)nc + 1) * sizeof(int), _st));
		YZ_LAUNCH(KColCount, GridFor(L.pnnz, kB), kB, 0, _st, L.pnnz, L.pcol.get(), _cnt.get());
		ScanExclusive(_cnt.get(), L.rptr.get(), nc, _scan.get(), _st);
		YZ_CUDA(cudaMemcpyAsync(_ifill.get(), L.rptr.get(), (size_t)nc * sizeof(int), cudaMemcpyDeviceToDevice, _st));
		YZ_LAUNCH(KTransposeFill, g, kB, 0, _st, n, L.pptr.get(), L.pcol.get(), L.pval.get(), _ifill.get(),
		          L.rcol.get(), L.rval.get());
		YZ_LAUNCH(KRowSort, GridFor((long long)nc * 32, 256, 148 * 64), 256, 0, _st, nc, L.rptr.get(), L.rcol.get(),
		          L.rval.get());
		//  AP, then A_c = R (AP)
		Gemm(n, L.ptr.get(), L.col.get(), L.val.get(), L.pptr.get(), L.pcol.get(), L.pval.get(), _apPtr, _apCol, _apVal);
		if(_levels.size() <= l + 1) _levels.emplace_back(new Level());
		_nlev = l + 2;
		Level &C = *_levels[l + 1];
		Level &F = *_levels[l];
		C.n = nc;
		C.nnz = Gemm(nc, F.rptr.get(), F.rcol.get(), F.rval.get(), _apPtr.get(), _apCol.get(), _apVal.get(), C.ptr, C.col,
		             C.val);
	}
	_haveH = true;
}

//  x = V(l) f from a zero guess
Sten Solver::StenOf(size_t l) const
{
	if(l == 0) return _sten;
	Sten none = Sten();
	return none;
}

void Solver::Cycle(size_t l, const double *f, double *x)
{
	Level &L = *_levels[l];
	const int n = L.n, g = GridFor(n, kB);
	if(L.direct)
	{
		YZ_LAUNCH(KDenseMV, GridFor((long long)n * 32, kB), kB, 0, _st, Halt(), n, L.inv.get(), f, x);
		return;
	}
	if(l + 1 < _nlev)
	{
		Level &C = *_levels[l + 1];
		YZ_LAUNCH(KPreSmoothResidual, g, kB, 0, _st, Halt(), n, L.ptr.get(), l == 0 ? _sellOff.get() : nullptr, StenOf(l),
		          l == 0 ? _sellCol.get() : L.col.get(), l == 0 ? _sellVal.get() : L.val.get(), L.M.get(), f, x, L.t.get());
		YZ_LAUNCH(KRestrict, GridFor((long long)C.n * 4, kB), kB, 0, _st, Halt(), C.n, L.rptr.get(), L.rcol.get(),
		          L.rval.get(), L.t.get(), C.f.get());
		Cycle(l + 1, C.f.get(), C.x.get());
		YZ_LAUNCH(KProlong, g, kB, 0, _st, Halt(), n, L.pptr.get(), L.pcol.get(), L.pval.get(), C.x.get(), x, L.xt.get());
		YZ_LAUNCH(KPostSmooth, g, kB, 0, _st, Halt(), n, L.ptr.get(), l == 0 ? _sellOff.get() : nullptr, StenOf(l),
		          l == 0 ? _sellCol.get() : L.col.get(), l == 0 ? _sellVal.get() : L.val.get(), L.M.get(), f, L.xt.get(), x);
	}
	else
	{
		YZ_LAUNCH(KPreSmooth, g, kB, 0, _st, Halt(), n, L.M.get(), f, L.xt.get());
		YZ_LAUNCH(KPostSmooth, g, kB, 0, _st, Halt(), n, L.ptr.get(), l == 0 ? _sellOff.get() : nullptr, StenOf(l),
		          l == 0 ? _sellCol.get() : L.col.get(), l == 0 ? _sellVal.get() : L.val.get(), L.M.get(), f, L.xt.get(), x);
	}
}

//  The same cycle in float (YZ_PREC_FP32_CYCLE) on the rounded copies that
//  RoundCycle made: f and x are the Krylov vectors (double) at the finest
//  level, the level's own float vectors below it.  The pre-smoothed x goes
//  to the level's x32 and the prolonged one to its xt32, so that the finest
//  level writes only the result into the caller's x.
template<class TF, class TX>
void Solver::Cycle32(size_t l, const TF *f, TX *x)
{
	Level &L = *_levels[l];
	const int n = L.n, g = GridFor(n, kB);
	if(L.direct)
	{
		YZ_LAUNCH_PDL((KDenseMV<float, TF, TX>), GridFor((long long)n * 32, kB), kB, 0, _st, Halt(), n, L.inv32.get(), f, x);
		return;
	}
	const int *so = l == 0 ? _sellOff.get() : nullptr, *col = l == 0 ? _sellCol.get() : L.col.get();
	const float *val = l == 0 ? _sellVal32.get() : L.val32.get();
	//  the finest level's smoothing around one persistent launch for all the
	//  coarser levels (yz_coarse.cuh)
	if(l == 0 && _nlev > 1 && CoarseCycleOn())
	{
		YZ_LAUNCH_PDL((KPreSmoothResidual<float, TF, float>), g, kB, 0, _st, Halt(), n, L.ptr.get(), so, StenOf(l), col,
		          val, L.M32.get(), f, L.x32.get(), L.t32.get());
		LaunchCoarseCycle();
		YZ_LAUNCH_PDL((KPostSmooth<float, TF, TX>), g, kB, 0, _st, Halt(), n, L.ptr.get(), so, StenOf(l), col, val,
		          L.M32.get(), f, L.xt32.get(), x);
		return;
	}
	if(l + 1 < _nlev)
	{
		Level &C = *_levels[l + 1];
		//  the coarse levels (CSR, float throughout) with several lanes a row
		constexpr bool coarse = std::is_same<TF, float>::value && std::is_same<TX, float>::value;
		if constexpr(coarse)
		{
			if((int)l >= FusedFrom())
			{
				CoarseDown(32, C.n, L, f, C.f32.get());
				Cycle32<float, float>(l + 1, C.f32.get(), C.x32.get());
				CoarseUp(std::max(2, LanesFor(L.nnz, n)), L, f, C.x32.get(), x);
				return;
			}
		}
		const int la = coarse ? LanesFor(L.nnz, n) : 1, lp = coarse ? LanesFor(L.pnnz, n) : 1;
		if constexpr(coarse)
		{
			if(la > 1) CoarsePreSmooth(la, n, L.ptr.get(), col, val, L.M32.get(), f, L.x32.get(), L.t32.get());
		}
		if(la == 1)
			YZ_LAUNCH_PDL((KPreSmoothResidual<float, TF, float>), g, kB, 0, _st, Halt(), n, L.ptr.get(), so, StenOf(l), col,
			          val, L.M32.get(), f, L.x32.get(), L.t32.get());
		YZ_LAUNCH_PDL(KRestrict<float>, GridFor((long long)C.n * 4, kB), kB, 0, _st, Halt(), C.n, L.rptr.get(), L.rcol.get(),
		          L.rval32.get(), L.t32.get(), C.f32.get());
		Cycle32<float, float>(l + 1, C.f32.get(), C.x32.get());
		if(lp > 1)
			CoarseProlong(lp, n, L.pptr.get(), L.pcol.get(), L.pval32.get(), C.x32.get(), L.x32.get(), L.xt32.get());
		else
			YZ_LAUNCH_PDL(KProlong<float>, g, kB, 0, _st, Halt(), n, L.pptr.get(), L.pcol.get(), L.pval32.get(), C.x32.get(),
			          L.x32.get(), L.xt32.get());
		if constexpr(coarse)
		{
			if(la > 1) CoarsePostSmooth(la, n, L.ptr.get(), col, val, L.M32.get(), f, L.xt32.get(), x);
		}
		if(la == 1)
		{
			//  FineSweeps() - 1 more SPAI0 sweeps at the finest level before
			//  the last, float to float (x32 and xt32 in turn)
			const float *xin = L.xt32.get();
			if(l == 0)
				for(int k = 1; k < FineSweeps(); ++k)
				{
					float *xo = (xin == L.xt32.get()) ? L.x32.get() : L.xt32.get();
					YZ_LAUNCH_PDL((KPostSmooth<float, TF, float>), g, kB, 0, _st, Halt(), n, L.ptr.get(), so, StenOf(l), col,
					          val, L.M32.get(), f, xin, xo);
					xin = xo;
				}
			YZ_LAUNCH_PDL((KPostSmooth<float, TF, TX>), g, kB, 0, _st, Halt(), n, L.ptr.get(), so, StenOf(l), col, val,
			          L.M32.get(), f, xin, x);
		}
	}
	else
	{
		YZ_LAUNCH_PDL((KPreSmooth<float, TF, float>), g, kB, 0, _st, Halt(), n, L.M32.get(), f, L.xt32.get());
		YZ_LAUNCH_PDL((KPostSmooth<float, TF, TX>), g, kB, 0, _st, Halt(), n, L.ptr.get(), so, StenOf(l), col, val, L.M32.get(), f,
		          L.xt32.get(), x);
	}
}

//  The persistent coarse cycle, switched on by YZ_COARSE_CYCLE=1 (while the
//  hierarchy has no more levels than the launch's plan holds).  Off by
//  default: on the 512^2 film its grid barriers cost more than the separate
//  launches they replace inside the loop's CUDA graph (65-69 against 80
//  steps/s with the FP32 V-cycle and reuse)
bool Solver::CoarseCycleOn() const
{
	static const char *env = std::getenv("YZ_COARSE_CYCLE");
	static const bool on = env && env[0] != '0';
	return on && _coarseOn && _nlev - 1 <= (size_t)kMaxCoarse;
}

//  blocks a multiprocessor of the persistent coarse cycle (YZ_COARSE_BLOCKS, default 1)
int Solver::CoarseBlocksPerSm()
{
	static const char *env = std::getenv("YZ_COARSE_BLOCKS");
	static const int k = env ? std::max(1, std::atoi(env)) : 1;
	return k;
}

void Solver::LaunchCoarseCycle()
{
	CoarsePlan P;
	const Level &F = *_levels[0];
	P.count = (int)_nlev - 1;
	P.n0 = F.n;
	P.p0Lanes = 1;
	P.t0 = F.t32.get(); P.x0 = F.x32.get(); P.xt0 = F.xt32.get();
	P.r0ptr = F.rptr.get(); P.r0col = F.rcol.get(); P.r0val = F.rval32.get();
	P.p0ptr = F.pptr.get(); P.p0col = F.pcol.get(); P.p0val = F.pval32.get();
	for(size_t l = 1; l < _nlev; ++l)
	{
		const Level &L = *_levels[l];
		CoarseLevel &c = P.lv[l - 1];
		c.n = L.n;
		c.direct = L.direct ? 1 : 0;
		c.last = (!L.direct && l + 1 == _nlev) ? 1 : 0;
		c.lanes = LanesFor(L.nnz, L.n);
		c.plLanes = LanesFor(L.pnnz, L.n);
		c.ptr = L.ptr.get(); c.col = L.col.get(); c.val = L.val32.get(); c.M = L.M32.get(); c.inv = L.inv32.get();
		c.f = L.f32.get(); c.x = L.x32.get(); c.t = L.t32.get(); c.xt = L.xt32.get();
		c.rptr = L.rptr.get(); c.rcol = L.rcol.get(); c.rval = L.rval32.get();
		c.pptr = L.pptr.get(); c.pcol = L.pcol.get(); c.pval = L.pval32.get();
	}
	if(_coarseBlocks == 0)
	{
		int occ = 0, sms = 0;
		YZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, KCoarseCycle, 256, 0));
		YZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, _device));
		_coarseBlocks = std::max(1, std::min(occ, CoarseBlocksPerSm())) * sms;
	}
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(_coarseBlocks);
	cfg.blockDim = dim3(256);
	cfg.dynamicSmemBytes = 0;
	cfg.stream = _st;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	const bool timed = TimedKernel("KCoarseCycle");
	if(timed) TimeBegin(_st);
	YZ_CUDA(cudaLaunchKernelEx(&cfg, KCoarseCycle, Halt(), P, _coarseBar.get(), _coarseErr.get()));
	if(timed) TimeEnd(_st);
	CountLaunches(1);
}

//  YZ_FUSE_FROM: the first level (1 or more) of the FP32 cycle whose way down
//  and way up each run as one launch; 0 switches the fused form off.  The
//  default, 2, is the measured best on the 512^2 film (four levels of
//  266,256 / ~30,000 / ~3,500 / ~400 rows): from level 1 the recomputation
//  costs what the launches save (the same solve time with a quarter fewer
//  launches), from level 2 the solve is 3 % faster than with no fusion.
//  SetTuning overrides it for one context.
int Solver::FusedFrom() const
{
	static const char *env = std::getenv("YZ_FUSE_FROM");
	static const int k = env ? (std::atoi(env) > 0 ? std::atoi(env) : 1 << 30) : 2;
	if(_fuseFrom == 0) return 1 << 30;
	return _fuseFrom > 0 ? _fuseFrom : k;
}

//  The FP32 cycle's post-smoothing sweeps at the finest level (the FP64
//  cycle keeps the reference's one).  SPAI0 smooths the film's fourth-order
//  rows weakly: on the 512^2 film 5 sweeps cut the BiCGStab iterations from
//  760 to 408 over 12 steps and the step from 11.7 to 9.7 ms (1: 85, 3: 99,
//  4: 101, 5: 102-103, 6-8: 101-102 steps/s).  YZ_FINE_SWEEPS or SetTuning
//  override the default, 5.
int Solver::FineSweeps() const
{
	static const char *env = std::getenv("YZ_FINE_SWEEPS");
	static const int k = env ? std::max(1, std::min(8, std::atoi(env))) : 5;
	return _fineSweeps > 0 ? _fineSweeps : k;
}

void Solver::SetTuning(int fuseFrom, int coarseLanes, int fineSweeps)
{
	if(fineSweeps < 0 || fineSweeps > 8) throw UsageError("set_tuning: fine_sweeps must be 0 (default) to 8");
	if(fuseFrom < -1) throw UsageError("set_tuning: fuse_from must be -1 (default), 0 (off) or a level >= 1");
	if(coarseLanes != 0 && coarseLanes != 1 && coarseLanes != 2 && coarseLanes != 4 && coarseLanes != 8)
		throw UsageError("set_tuning: coarse_lanes must be 0 (by row length), 1, 2, 4 or 8");
	if(fuseFrom != _fuseFrom || coarseLanes != _coarseLanes || fineSweeps != _fineSweeps)
		++_epoch;   // the loop graph holds the old shapes
	_fuseFrom = fuseFrom;
	_coarseLanes = coarseLanes;
	_fineSweeps = fineSweeps;
}

//  lanes a row for a coarse level of the FP32 cycle, by its mean row length
int Solver::LanesFor(long long nnz, int n) const
{
	if(_coarseLanes > 0) return _coarseLanes;
	const long long avg = n > 0 ? nnz / n : 0;
	return avg >= 24 ? 8 : avg >= 10 ? 4 : avg >= 4 ? 2 : 1;
}

#define YZ_BY_LANES(lanes, K, n, ...)                                                                   \
	do {                                                                                                \
		switch(lanes)                                                                                   \
		{                                                                                               \
		case 8:  YZ_LAUNCH_PDL((K<8, float>), GridFor((long long)(n) * 8, kB), kB, 0, _st, __VA_ARGS__); break;  \
		case 4:  YZ_LAUNCH_PDL((K<4, float>), GridFor((long long)(n) * 4, kB), kB, 0, _st, __VA_ARGS__); break;  \
		default: YZ_LAUNCH_PDL((K<2, float>), GridFor((long long)(n) * 2, kB), kB, 0, _st, __VA_ARGS__); break;  \
		}                                                                                               \
	} while(0)

void Solver::CoarsePreSmooth(int lanes, int n, const int *ptr, const int *col, const float *val, const float *M,
                             const float *f, float *x, float *t)
{
	YZ_BY_LANES(lanes, KPreSmoothResidualL, n, Halt(), n, ptr, col, val, M, f, x, t);
}

void Solver::CoarsePostSmooth(int lanes, int n, const int *ptr, const int *col, const float *val, const float *M,
                              const float *f, const float *x, float *xout)
{
	YZ_BY_LANES(lanes, KPostSmoothL, n, Halt(), n, ptr, col, val, M, f, x, xout);
}

void Solver::CoarseProlong(int lanes, int n, const int *pptr, const int *pcol, const float *pval, const float *xc,
                           const float *x, float *xout)
{
	YZ_BY_LANES(lanes, KProlongL, n, Halt(), n, pptr, pcol, pval, xc, x, xout);
}
void Solver::CoarseDown(int lanes, int nc, const Level &L, const float *f, float *fc)
{
	if(lanes == 32)
		YZ_LAUNCH_PDL((KDownFused<32, float>), GridFor((long long)nc * 32, kB), kB, 0, _st, Halt(), nc, L.rptr.get(),
		          L.rcol.get(), L.rval32.get(), L.ptr.get(), L.col.get(), L.val32.get(), L.M32.get(), f, fc);
	else
		YZ_BY_LANES(lanes, KDownFused, nc, Halt(), nc, L.rptr.get(), L.rcol.get(), L.rval32.get(), L.ptr.get(),
		            L.col.get(), L.val32.get(), L.M32.get(), f, fc);
}

void Solver::CoarseUp(int lanes, const Level &L, const float *f, const float *xc, float *x)
{
	YZ_BY_LANES(lanes, KUpFused, L.n, Halt(), L.n, L.ptr.get(), L.col.get(), L.val32.get(), L.M32.get(), L.pptr.get(),
	            L.pcol.get(), L.pval32.get(), f, xc, x);
}
#undef YZ_BY_LANES

//  After an FP64 set-up: every level's matrices rounded to float for
//  Cycle32 (the finest level's A was rounded by KScaleGather), in one launch
void Solver::RoundCycle()
{
	RoundList list;
	list.count = 0;
	auto add = [&](const double *src, float *dst, long long cnt) {
		if(cnt <= 0) return;
		if(list.count == RoundList::kMax)
		{
			YZ_LAUNCH(KRoundToFloat, 148 * 4, kB, 0, _st, list);
			list.count = 0;
		}
		list.src[list.count] = src; list.dst[list.count] = dst; list.n[list.count] = cnt; ++list.count;
	};
	for(size_t l = 0; l < _nlev; ++l)
	{
		Level &L = *_levels[l];
		const size_t n = (size_t)L.n;
		L.f32.reserve(n); L.x32.reserve(n); L.t32.reserve(n); L.xt32.reserve(n);
		if(L.direct)
		{
			L.inv32.reserve(n * n);
			add(L.inv.get(), L.inv32.get(), (long long)(n * n));
			continue;
		}
		L.M32.reserve(n);
		add(L.M.get(), L.M32.get(), (long long)n);
		if(l > 0)
		{
			L.val32.reserve((size_t)L.nnz);
			add(L.val.get(), L.val32.get(), L.nnz);
		}
		if(l + 1 < _nlev)
		{
			L.pval32.reserve((size_t)L.pnnz); L.rval32.reserve((size_t)L.pnnz);
			add(L.pval.get(), L.pval32.get(), L.pnnz);
			add(L.rval.get(), L.rval32.get(), L.pnnz);
		}
	}
	if(list.count) YZ_LAUNCH(KRoundToFloat, 148 * 4, kB, 0, _st, list);
}

void Solver::SetPrecision(int precision)
{
	if(precision != YZ_PREC_FP64 && precision != YZ_PREC_FP32_CYCLE && precision != YZ_PREC_FP32_MATRIX)
		throw UsageError("set_precision: precision must be YZ_PREC_FP64, YZ_PREC_FP32_CYCLE or YZ_PREC_FP32_MATRIX");
	if(precision != _precision)
	{
		++_epoch;
		//  a hierarchy set up in the other precision has no (or stale)
		//  float copies: the next AMG solve sets up afresh
		_stale = true;
	}
	_precision = precision;
}

void Solver::SetAmgReuse(int maxSolves)
{
	if(maxSolves < 0) throw UsageError("set_amg_reuse: max_solves must be >= 0");
	_amgReuse = maxSolves;
	_sinceBuild = 0;
	_stale = true;		// the next AMG solve sets up afresh
}

void Solver::SetLearned(Learned *L, int mode, int collectSolves, int perSolve, double capFactor)
{
	if(mode < 0 || mode > 2) throw UsageError("set_learned: mode must be 0 (off), 1 (collect) or 2 (use)");
	if(mode && !L) throw UsageError("set_learned: no network given");
	if(L && _n > 0 && L->Rows() != _n) throw UsageError("set_learned: the network's grid does not have the pattern's rows");
	if(capFactor <= 0) throw UsageError("set_learned: cap_factor must be > 0");
	if(L != _learned) ++_epoch;
	_learned = L;
	_learnedMode = mode;
	_collectLeft = (mode >= 1) ? collectSolves : 0;
	_perSolve = perSolve;
	_capFactor = capFactor;
	_offLearned = TryBackoff();
}

void Solver::ApplyPrec(int kind, const double *r, double *z)
{
	const int n = _n;
	if(kind == kPrecLearned) { _learned->Apply(r, z, _st, Halt()); return; }
	if(kind == kPrecDiag) YZ_LAUNCH(KDiagApply, GridFor(n, kB), kB, 0, _st, Halt(), n, _m.get(), r, z);
	else if(_precision != YZ_PREC_FP64) Cycle32<double, double>(0, r, z);
	else Cycle(0, r, z);
}

//  One BiCGStab iteration queued on the stream: every kernel reads the run's
//  state word and does nothing once it is set (KState), so iterations may be
//  queued ahead of the test the host would make between them.
void Solver::EnqueueIteration(int kind)
{
	Level &A = *_levels[0];
	const int n = _n, nb = RedBlocks(n), g = GridFor(n, kB);
	const int *ptr = A.ptr.get(), *so = _sellOff.get(), *col = _sellCol.get();
	const double *val = _sellVal.get();
	//  YZ_PREC_FP32_MATRIX: the SpMVs read the float copy of the values
	const float *val32 = _precision == YZ_PREC_FP32_MATRIX ? _sellVal32.get() : nullptr;
	Scal *sc = _sc.get();
	double *x = _x.get();
	YZ_LAUNCH_PDL(KPUpdate, g, kB, 0, _st, n, _r.get(), _v.get(), _p.get(), sc);
	ApplyPrec(kind, _p.get(), _ph.get());
	if(val32)
		YZ_LAUNCH_PDL(KSpmvAlpha<float>, nb, kRT, 0, _st, n, ptr, so, _sten, col, val32, _ph.get(), _rh.get(), _v.get(), Red(1), sc);
	else
		YZ_LAUNCH_PDL(KSpmvAlpha<double>, nb, kRT, 0, _st, n, ptr, so, _sten, col, val, _ph.get(), _rh.get(), _v.get(), Red(1), sc);
	YZ_LAUNCH_PDL(KSUpdate, nb, kRT, 0, _st, n, _r.get(), _v.get(), _s.get(), Red(2), sc);
	ApplyPrec(kind, _s.get(), _sh.get());
	if(val32)
		YZ_LAUNCH_PDL(KSpmvOmega<float>, nb, kRT, 0, _st, n, ptr, so, _sten, col, val32, _sh.get(), _s.get(), _t.get(), Red(3), sc);
	else
		YZ_LAUNCH_PDL(KSpmvOmega<double>, nb, kRT, 0, _st, n, ptr, so, _sten, col, val, _sh.get(), _s.get(), _t.get(), Red(3), sc);
	YZ_LAUNCH_PDL(KXRUpdate, nb, kRT, 0, _st, n, _ph.get(), _sh.get(), _s.get(), _t.get(), _rh.get(), x, _r.get(),
	          Red(4), sc);
}

//  The iterations of one run until its state is set, as one CUDA graph
//  launch and one read of the state, or from the stream with one iteration
//  kept in flight (the host's test between two iterations of the oracle is
//  on the device either way).
void Solver::RunIterations(int kind)
{
	//  The loop runs as a CUDA graph: a conditional while node whose body is
	//  one iteration, so that the device decides when it ends and the host
	//  launches nothing per iteration.  The graph is kept while its kernels
	//  and buffers stay those it was captured with (the same pattern and
	//  precision and, for the AMG kind, the same hierarchy: a reused one),
	//  and captured anew otherwise (0.2-0.5 ms, less than the host launches
	//  it saves on the 512^2 film).  YZ_GRAPH=0, the context's switch off
	//  (SetGraphLoop), or a kernel being timed: the iterations are launched
	//  from the stream instead.
	static const char *env = std::getenv("YZ_GRAPH");
	static const bool graphOff = env && env[0] == '0';
	LoopGraph &lg = _loop[kind];
	const unsigned long long key = ((unsigned long long)_epoch << 32) | (kind == kPrecAmg ? _epochH : 0u);
	Scal *sc = _sc.get();
	//  an AMG run that feeds the network's sample ring: after each of its
	//  first iterations, the residual r and the V-cycle's answer to it
	const bool collect = kind == kPrecAmg && _learned && _filmSolve && _collectLeft > 0 && _perSolve > 0;
	int hooks = 0;
	auto hook = [&]() {
		if(!collect || hooks >= _perSolve) return;
		ApplyPrec(kPrecAmg, _r.get(), _zs.get());
		_learned->AddSample(_r.get(), _zs.get(), _st, Halt());
		++hooks;
	};
	if(collect) _zs.reserve((size_t)_n);
	if(graphOff || !_graphLoop || TimingActive() || collect)
	{
		//  one iteration kept in flight: the state after iteration k is
		//  copied to pinned memory and read while iteration k+1 runs; the
		//  iteration queued after the last one finds the state set and does
		//  nothing.  While a kernel is timed, the timed launches of the
		//  iterations that found the run stopped are dropped: an iteration
		//  launches the timed kernel the same number of times each, and the
		//  iterations that did work are the run's count (exact for a kernel
		//  that precedes the half-step test, as KSpmvAlpha).
		const long long mark = TimeCount();
		_tailDone = false;		// Solve copies the answer after this run
		int queued = 0;
		int slot = 0;
		hook();			// the start residual r = b - A x0
		EnqueueIteration(kind); ++queued;
		YZ_LAUNCH(KLoopCount, 1, 1, 0, _st, sc);
		hook();
		YZ_CUDA(cudaMemcpyAsync(_hring + slot, sc, sizeof(Scal), cudaMemcpyDeviceToHost, _st));
		YZ_CUDA(cudaEventRecord(_evRing[slot], _st));
		for(;;)
		{
			EnqueueIteration(kind); ++queued;
			YZ_LAUNCH(KLoopCount, 1, 1, 0, _st, sc);
			hook();
			const int next = slot ^ 1;
			YZ_CUDA(cudaMemcpyAsync(_hring + next, sc, sizeof(Scal), cudaMemcpyDeviceToHost, _st));
			YZ_CUDA(cudaEventRecord(_evRing[next], _st));
			YZ_CUDA(cudaEventSynchronize(_evRing[slot]));
			const Scal &h = _hring[slot];
			if(h.state != kRun || h.it >= h.maxIter)
			{
				YZ_CUDA(cudaStreamSynchronize(_st));
				*_hsc = h;
				break;
			}
			slot = next;
		}
		const long long timed = TimeCount() - mark;
		if(timed > 0 && queued > _hsc->it) TimeDropLast(timed / queued * (queued - _hsc->it));
		if(collect) { --_collectLeft; _collected += hooks; }
		return;
	}
	if(lg.exec == nullptr || lg.key != key)
	{
		FreeLoopGraph(lg);
		BuildLoopGraph(kind, lg);
		lg.key = key;
	}
	YZ_CUDA(cudaGraphLaunch(lg.exec, _st));
	//  the end of the run queued behind the loop -- its time, the answer
	//  into the caller's x (Solve's tail) -- so that one wait covers all
	YZ_CUDA(cudaEventRecord(_ev2, _st));
	if(_tailDst)
	{
		YZ_CUDA(cudaMemcpyAsync(_tailDst, _tailSrc, _tailBytes, cudaMemcpyDeviceToDevice, _st));
		_tailDone = true;
	}
	ReadScal();
	//  the kernels the loop ran
	CountLaunches(lg.perBody * (long long)_hsc->bodies);
}

void Solver::FreeLoopGraph(LoopGraph &g)
{
	if(g.exec) cudaGraphExecDestroy(g.exec);
	if(g.graph) cudaGraphDestroy(g.graph);
	g.exec = nullptr;
	g.graph = nullptr;
	g.key = ~0ull;
}

void Solver::BuildLoopGraph(int kind, LoopGraph &lg)
{
	Scal *sc = _sc.get();
	cudaGraph_t graph = nullptr, body = nullptr;
	cudaGraphExec_t exec = nullptr;
	YZ_CUDA(cudaGraphCreate(&graph, 0));
	try
	{
		cudaGraphConditionalHandle h;
		YZ_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
		//  the other members are value-initialised (zero), as the API asks
		cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
		cp.conditional.handle = h;
		cp.conditional.type = cudaGraphCondTypeWhile;
		cp.conditional.size = 1;
		cudaGraphNode_t node;
		YZ_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
		body = cp.conditional.phGraph_out[0];
		const long long l0 = t_launches;
		YZ_CUDA(cudaStreamBeginCaptureToGraph(_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
		try
		{
			EnqueueIteration(kind);
			YZ_LAUNCH(KLoopCond, 1, 1, 0, _st, h, sc);
		}
		catch(...)
		{
			cudaGraph_t dummy = nullptr;
			cudaStreamEndCapture(_st, &dummy);
			throw;
		}
		YZ_CUDA(cudaStreamEndCapture(_st, &body));
		lg.perBody = t_launches - l0;
		CountLaunches(-lg.perBody);
		YZ_CUDA(cudaGraphInstantiate(&exec, graph, 0));
	}
	catch(...)
	{
		if(exec) cudaGraphExecDestroy(exec);
		cudaGraphDestroy(graph);
		throw;
	}
	lg.graph = graph;
	lg.exec = exec;
}

//  BiCGStab on level 0's matrix (values in _levels[0]); the oracle's
//  BiCGStab() step by step.  The start tests run on the device (KCtlStart),
//  so the host waits once, after the run (RunIterations leaves the state in
//  _hsc).  Returns false on a breakdown (rho == 0).
bool Solver::BiCGStab(int kind, int maxIter, double tol, int &itOut, double &errOut)
{
	Level &A = *_levels[0];
	const int n = _n, nb = RedBlocks(n), g = GridFor(n, kB);
	double *b = _b.get(), *x = _x.get();
	if(_precision == YZ_PREC_FP32_MATRIX)
		YZ_LAUNCH(KBInit, nb, kRT, 0, _st, n, A.ptr.get(), _sellOff.get(), _sten, _sellCol.get(),
		          (const float *)_sellVal32.get(), b, x, _r.get(), _rh.get(), Red(0), _sc.get());
	else
		YZ_LAUNCH(KBInit, nb, kRT, 0, _st, n, A.ptr.get(), _sellOff.get(), _sten, _sellCol.get(), _sellVal.get(), b, x,
		          _r.get(), _rh.get(), Red(0), _sc.get());
	YZ_LAUNCH(KCtlStart, 1, 1, 0, _st, _sc.get(), tol, maxIter);
	YZ_LAUNCH(KZeroIfTiny, g, kB, 0, _st, n, _sc.get(), x);
	RunIterations(kind);
	const Scal &h = *_hsc;
	if(h.state == kTiny) { itOut = 0; errOut = h.normb; return true; }
	if(h.state == kBreak) return false;
	itOut = (h.state == kSkip) ? 0 : h.it;
	errOut = h.res / h.normb;
	return true;
}

//  LinearSolverBackend.cpp:681-713, on the host (a breakdown is rare): the
//  residual of what x holds, summed sequentially as the reference does
double Solver::BreakdownResidual()
{
	const int n = _n, nnz = _nnz;
	std::vector<double> val((size_t)nnz), b((size_t)n), x((size_t)n);
	_levels[0]->val.download(val.data(), (size_t)nnz, _st);
	_b.download(b.data(), (size_t)n, _st);
	_x.download(x.data(), (size_t)n, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
	double rr = 0.0, bb = 0.0;
	for(int i = 0; i < n; ++i)
	{
		double ax = 0.0;
		for(int k = _hptr[(size_t)i]; k < _hptr[(size_t)i + 1]; ++k) ax += val[(size_t)k] * x[(size_t)_hcol[(size_t)k]];
		const double d = b[(size_t)i] - ax;
		rr += d * d; bb += b[(size_t)i] * b[(size_t)i];
	}
	return (bb > 0.0) ? std::sqrt(rr / bb) : std::sqrt(rr);
}

int Solver::Solve(const yz_settings &set, const double *dValues, const double *dRhs, double *dX, int &iterOut, double &residOut)
{
	if(_n <= 0) throw UsageError("solve: set_pattern first");
	if(set.max_iteration < 0) throw UsageError("solve: max_iteration must be >= 0");
	YZ_CUDA(cudaSetDevice(_device));
	const long long l0 = t_launches;
	const int n = _n, nnz = _nnz, g = GridFor(n, kB);
	Level &L0 = *_levels[0];
	const bool fp32 = _precision != YZ_PREC_FP64;
	if(fp32)
	{
		const float *was = _sellVal32.get();
		_sellVal32.reserve(_sellSize);
		if(_sellVal32.get() != was) ++_epoch;
	}
	{
		YZ_PROF("lin.prepare", _st);
		YZ_LAUNCH(KScaleGather, g, kB, 0, _st, n, L0.ptr.get(), _ssrc.get(), dValues, dRhs, set.scaling ? 1 : 0,
		          L0.val.get(), _b.get(), _sellOff.get(), _sellVal.get(), fp32 ? _sellVal32.get() : nullptr);
		(void)nnz;
		YZ_CUDA(cudaMemcpyAsync(_x.get(), dX, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
		YZ_CUDA(cudaMemcpyAsync(_x0.get(), dX, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
	}
	//  a film solve that collects training pairs stores them with the
	//  features of its own system (the matrix diagonal and the film height),
	//  those the network reads when it is applied to such a system
	_filmSolve = !set.conc && set.precondition == 2;
	if(_learned && _filmSolve && _collectLeft > 0 && _perSolve > 0) _learned->SetAux(dValues, L0.ptr.get(), _aux, _st);
	YZ_CUDA(cudaEventRecord(_ev0, _st));
	//  a run in graph form copies its answer to dX behind the loop (the
	//  last run's copy is the one that stays)
	_tailDst = dX; _tailSrc = _x.get(); _tailBytes = (size_t)n * sizeof(double); _tailDone = false;
	_setupMs = 0; _iterMs = 0;
	int it = 0, itTried = 0;
	double err = 0.0;
	const int tryIter = set.max_iteration < 300 ? set.max_iteration : 300;
	bool done = false;
	bool timedSetup = false;

	if(set.conc && set.precondition == 2 && _offSpai.Try())
	{
		YZ_PROF("lin.fallback.conc", _st);
		YZ_LAUNCH(KSpai0, g, kB, 0, _st, n, L0.ptr.get(), L0.col.get(), L0.val.get(), _m.get());
		if(!BiCGStab(kPrecDiag, tryIter, set.epsilon, it, err)) err = 1e300;
		if(err <= set.epsilon) { done = true; _offSpai.Converged(); }
		else
		{
			_offSpai.Failed();
			itTried = it;
			YZ_CUDA(cudaMemcpyAsync(_x.get(), _x0.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
		}
	}
	//  The learned preconditioner first, on a solve of the film (SA-AMG
	//  preconditioning asked for, not the concentration's role): a flexible
	//  BiCGStab (the right-preconditioned iteration with the network as its
	//  preconditioner, which may change from one application to the next;
	//  x and the residual recurrence stay those of the true matrix) allowed
	//  cap_factor times the last SA-AMG solve's iterations.  One that does not
	//  converge within them is repeated from the caller's guess on the AMG
	//  path, and the network sits out the next solves (TryBackoff, as the
	//  SPAI0 try does).
	if(!done && _learnedMode == 2 && _learned && _learned->Trained() && !set.conc && set.precondition == 2)
	{
		if(_offLearned.Try())
		{
			YZ_PROF("lin.learned", _st);
			_learned->SetAux(dValues, L0.ptr.get(), _aux, _st);
			//  the plain path's count: the last SA-AMG solve's, else the cap
			const double plain = _amgIters > 0 ? (double)_amgIters : (double)set.max_iteration;
			const int cap = (int)std::max(1.0, std::min((double)set.max_iteration, std::ceil(_capFactor * plain)));
			int itL = 0;
			double errL = 0;
			const bool okL = BiCGStab(kPrecLearned, cap, set.epsilon, itL, errL);
			if(okL && errL <= set.epsilon)
			{
				done = true; it = itL; err = errL;
				++_lstats.solves; _lstats.iterations += itL;
				_offLearned.Converged();
			}
			else
			{
				++_lstats.fallbacks;
				itTried += okL ? itL : 0;
				_offLearned.Failed();
				YZ_CUDA(cudaMemcpyAsync(_x.get(), _x0.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
			}
		}
		else
			++_lstats.skipped;
	}
	bool broke = false;
	if(!done && FaultNow()) broke = true;
	else if(!done)
	{
		if(set.precondition == 0 || set.precondition == 1)
		{
			{
				YZ_PROF("lin.precond", _st);
				YZ_LAUNCH(KDiag, g, kB, 0, _st, n, L0.ptr.get(), L0.col.get(), L0.val.get(), _dia.get());
				YZ_LAUNCH(KDampedJacobi, g, kB, 0, _st, n, _dia.get(), _m.get());
			}
			YZ_PROF("lin.iterate", _st);
			broke = !BiCGStab(kPrecDiag, set.max_iteration, set.epsilon, it, err);
		}
		else
		{
			//  with reuse on, the last set-up's hierarchy serves until it has
			//  served _amgReuse solves or a solve on it took clearly more
			//  iterations than the first one did; only the finest level's
			//  SPAI0 is recomputed from the new matrix (the finest level's A
			//  in the cycle is the new matrix itself)
			for(;;)
			{
				//  a float cycle runs only on a hierarchy that has its float
				//  copies (one set up, or rounded, in a float precision)
				const bool reuse = _amgReuse > 0 && _haveH && !_stale && _sinceBuild < _amgReuse &&
				                   (!fp32 || _hPrec != YZ_PREC_FP64);
				{
					YZ_PROF("lin.precond", _st);
					if(reuse)
					{
						Level &F = *_levels[0];
						if(!F.direct)
						{
							YZ_LAUNCH(KSpai0, g, kB, 0, _st, n, F.ptr.get(), F.col.get(), F.val.get(), F.M.get());
							if(fp32)
							{
								RoundList one;
								one.count = 1; one.src[0] = F.M.get(); one.dst[0] = F.M32.get(); one.n[0] = n;
								YZ_LAUNCH(KRoundToFloat, GridFor(n, kB), kB, 0, _st, one);
							}
						}
						++_sinceBuild;
					}
					else
					{
						BuildHierarchy(n > 3000 ? 500 : 3000);
						if(fp32) RoundCycle();
						_hPrec = _precision;
						_sinceBuild = 0;
						_stale = false;
					}
				}
				YZ_CUDA(cudaEventRecord(_ev1, _st));
				timedSetup = true;
				{
					YZ_PROF("lin.iterate", _st);
					broke = !BiCGStab(kPrecAmg, set.max_iteration, set.epsilon, it, err);
				}
				if(!broke && !set.conc && err <= set.epsilon) _amgIters = it;
				if(!reuse) { _freshIters = it; break; }
				if(broke || !(err <= set.epsilon))
				{
					//  the old hierarchy failed where a new one may not: set up
					//  afresh and solve again from the caller's guess
					_stale = true;
					itTried += broke ? 0 : it;
					YZ_CUDA(cudaMemcpyAsync(_x.get(), _x0.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
					continue;
				}
				if(it > _freshIters + std::max(4, _freshIters / 2)) _stale = true;
				break;
			}
		}
	}
	_tailDst = nullptr;
	if(!_tailDone) YZ_CUDA(cudaEventRecord(_ev2, _st));	// else recorded behind the loop
	YZ_CUDA(cudaEventSynchronize(_ev2));
	if(fp32 && CoarseCycleOn())
	{
		int e = 0;
		YZ_CUDA(cudaMemcpy(&e, _coarseErr.get(), sizeof(int), cudaMemcpyDeviceToHost));
		if(e) throw CudaError("solve: a grid barrier of the coarse V-cycle timed out");
	}
	float ms = 0;
	if(timedSetup)
	{
		YZ_CUDA(cudaEventElapsedTime(&ms, _ev0, _ev1)); _setupMs = ms;
		YZ_CUDA(cudaEventElapsedTime(&ms, _ev1, _ev2)); _iterMs = ms;
	}
	else { YZ_CUDA(cudaEventElapsedTime(&ms, _ev0, _ev2)); _iterMs = ms; }
	_launches += t_launches - l0;
	if(broke)
	{
		const double rel = BreakdownResidual();
		if(rel <= set.epsilon && rel == rel) { it = 0; err = rel; }
		else
		{
			//  x is left as the caller gave it
			if(_tailDone)
			{
				YZ_CUDA(cudaMemcpyAsync(dX, _x0.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
				YZ_CUDA(cudaStreamSynchronize(_st));
			}
			iterOut = itTried; residOut = rel; return 2;
		}
	}
	if(!_tailDone)
	{
		YZ_CUDA(cudaMemcpyAsync(dX, _x.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, _st));
		YZ_CUDA(cudaStreamSynchronize(_st));
	}
	iterOut = it + itTried;
	residOut = err;
	if(err <= set.epsilon) return 0;
	if(!(err == err)) return 2;
	return 1;
}

int Solver::SolveHost(const yz_settings &set, const double *values, const double *rhs, double *x, int &iter, double &resid)
{
	if(_n <= 0) throw UsageError("solve: set_pattern first");
	YZ_CUDA(cudaSetDevice(_device));
	_values.upload(values, (size_t)_nnz, _st);
	_rhs.upload(rhs, (size_t)_n, _st);
	_xio.upload(x, (size_t)_n, _st);
	const int ret = Solve(set, _values.get(), _rhs.get(), _xio.get(), iter, resid);
	if(ret != 2)
	{
		_xio.download(x, (size_t)_n, _st);
		YZ_CUDA(cudaStreamSynchronize(_st));
	}
	return ret;
}

std::vector<double> Solver::Memory() const { return {(double)_offSpai.skip, (double)_offSpai.wait}; }
void Solver::SetMemory(const double *m, int len)
{
	if(len != 2) return;
	_offSpai.skip = (int)m[0]; _offSpai.wait = (int)m[1];
}

int Solver::LevelCount() const { return _haveH ? (int)_nlev : 0; }

void Solver::LevelInfo(int l, int *rows, int *nnzA, int *nnzP, int *direct) const
{
	if(!_haveH || l < 0 || l >= (int)_nlev) throw UsageError("level_info: no such level");
	const Level &L = *_levels[(size_t)l];
	if(rows) *rows = L.n;
	if(nnzA) *nnzA = L.nnz;
	if(nnzP) *nnzP = (L.direct || L.nc == 0) ? 0 : L.pnnz;
	if(direct) *direct = L.direct ? 1 : 0;
}

void Solver::LevelCopy(int l, int *aptr, int *acol, double *aval, int *pptr, int *pcol, double *pval, int *agg)
{
	if(!_haveH || l < 0 || l >= (int)_nlev) throw UsageError("level_copy: no such level");
	YZ_CUDA(cudaSetDevice(_device));
	Level &L = *_levels[(size_t)l];
	if(aptr) L.ptr.download(aptr, (size_t)L.n + 1, _st);
	if(acol) L.col.download(acol, (size_t)L.nnz, _st);
	if(aval) L.val.download(aval, (size_t)L.nnz, _st);
	if(!L.direct && L.nc > 0)
	{
		if(pptr) L.pptr.download(pptr, (size_t)L.n + 1, _st);
		if(pcol) L.pcol.download(pcol, (size_t)L.pnnz, _st);
		if(pval) L.pval.download(pval, (size_t)L.pnnz, _st);
	}
	if(agg && !L.direct) L.agg.download(agg, (size_t)L.n, _st);
	YZ_CUDA(cudaStreamSynchronize(_st));
}

//--------------------------------------------------------------------------
//  stand-alone building blocks
//--------------------------------------------------------------------------
double DeviceDot(int n, const double *hx, const double *hy)
{
	DBuf<double> x, y, part, out;
	DBuf<unsigned> cnt;
	x.upload(hx, (size_t)n, 0); y.upload(hy, (size_t)n, 0);
	const int nb = RedBlocks(n);
	part.reserve((size_t)nb); out.reserve(1); cnt.reserve(1);
	YZ_CUDA(cudaMemset(cnt.get(), 0, sizeof(unsigned)));
	RedScratch rs{part.get(), cnt.get(), nb};
	YZ_LAUNCH(KDot, nb, kRT, 0, 0, n, x.get(), y.get(), rs, out.get());
	double h = 0;
	YZ_CUDA(cudaMemcpy(&h, out.get(), sizeof(double), cudaMemcpyDeviceToHost));
	return h;
}

void DeviceSpmv(int n, int nnz, const int *rowptr, const int *col, const double *val, const double *hx, double *hy)
{
	DBuf<int> p, c; DBuf<double> v, x, y;
	p.upload(rowptr, (size_t)n + 1, 0); c.upload(col, (size_t)nnz, 0); v.upload(val, (size_t)nnz, 0);
	x.upload(hx, (size_t)n, 0); y.reserve((size_t)n);
	YZ_LAUNCH(KSpmv, GridFor(n, kB), kB, 0, 0, nullptr, n, p.get(), c.get(), v.get(), x.get(), y.get());
	YZ_CUDA(cudaMemcpy(hy, y.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
}

} // namespace yz
