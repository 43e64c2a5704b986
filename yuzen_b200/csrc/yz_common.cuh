// yz_common.cuh -- shared host/device utilities of the B200 implicit-step library.
//
// Built for sm_100a only.  The FP64 parity kernels are compiled with
// -fmad=false so that every a*b+c rounds twice, as the reference's host code
// does under -ffp-contract=off (CMakeLists.txt:33-46).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace yz {

//--------------------------------------------------------------------------
//  errors and launch accounting
//--------------------------------------------------------------------------
struct CudaError : std::runtime_error
{
	explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};
struct UsageError : std::runtime_error
{
	explicit UsageError(const std::string &m) : std::runtime_error(m) {}
};
//  a numerical failure of the time step (the reference's FatalError at the
//  step: dt below MinDt, ImplicitSolver.cpp:180-184; no convergence at a
//  fixed step, FailedFixedStep, ImplicitSolver.cpp:192-201)
struct StepFailed : std::runtime_error
{
	explicit StepFailed(const std::string &m) : std::runtime_error(m) {}
};

inline void Check(cudaError_t e, const char *what)
{
	if(e != cudaSuccess)
	{
		//  a failed call also leaves its error as the thread's last error:
		//  take it, so that the next launch's check does not report it again
		(void)cudaGetLastError();
		throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
	}
}
#define YZ_CUDA(call) ::yz::Check((call), #call)

//  Every kernel launch of the library goes through YZ_LAUNCH, which counts it,
//  and, for the one kernel named by yz_time_kernel(), brackets it with CUDA
//  events on its own stream (the per-launch device time of that kernel).
extern std::atomic<long long> g_launches;     // every launch of the process (yz_launch_count)
extern thread_local long long t_launches;     // this thread's: a context's counts are taken from it
//  count n launches (negative: take back launches that were captured, not run)
inline void CountLaunches(long long n)
{
	g_launches.fetch_add(n, std::memory_order_relaxed);
	t_launches += n;
}
bool TimedKernel(const char *name);
bool TimingActive();   // a kernel is selected for per-launch timing
void TimeBegin(cudaStream_t st);
void TimeEnd(cudaStream_t st);
long long TimeCount();            // timed launches recorded so far
void TimeDropLast(long long k);   // forget the last k of them

#define YZ_LAUNCH(kernel, grid, block, smem, stream, ...)                         \
	do {                                                                          \
		const bool yzTimed_ = ::yz::TimedKernel(#kernel);                         \
		if(yzTimed_) ::yz::TimeBegin(stream);                                     \
		kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);               \
		if(yzTimed_) ::yz::TimeEnd(stream);                                       \
		::yz::CountLaunches(1);                                                   \
		::yz::Check(cudaGetLastError(), #kernel);                                 \
	} while(0)

//  Programmatic dependent launch for the chains of short kernels in the
//  BiCGStab loop and the V-cycle: a kernel launched by YZ_LAUNCH_PDL may be
//  scheduled while the kernel before it on the stream drains.  Such a kernel
//  begins with PdlEntry(): griddepcontrol.wait holds every thread until the
//  kernels it depends on have completed and their memory is visible (so its
//  reads and writes are those of a plain launch), then launch_dependents lets
//  the next kernel be scheduled.  Without the launch attribute both are no-ops.
//  YZ_PDL=0 in the environment launches these kernels plainly.
bool PdlOn();
__device__ __forceinline__ void PdlEntry()
{
#if defined(__CUDA_ARCH__)
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}
#define YZ_LAUNCH_PDL(kernel, grid, block, smem, strm, ...)                     \
	do {                                                                          \
		const bool yzTimed_ = ::yz::TimedKernel(#kernel);                         \
		if(yzTimed_) ::yz::TimeBegin(strm);                                     \
		if(::yz::PdlOn())                                                         \
		{                                                                         \
			cudaLaunchConfig_t yzCfg_ = {};                                       \
			yzCfg_.gridDim = dim3(grid);                                          \
			yzCfg_.blockDim = dim3(block);                                        \
			yzCfg_.dynamicSmemBytes = (smem);                                     \
			yzCfg_.stream = (strm);                                             \
			cudaLaunchAttribute yzAttr_[1];                                       \
			yzAttr_[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;   \
			yzAttr_[0].val.programmaticStreamSerializationAllowed = 1;            \
			yzCfg_.attrs = yzAttr_;                                               \
			yzCfg_.numAttrs = 1;                                                  \
			::yz::Check(cudaLaunchKernelEx(&yzCfg_, kernel, __VA_ARGS__), #kernel); \
		}                                                                         \
		else                                                                      \
			kernel<<<(grid), (block), (smem), (strm)>>>(__VA_ARGS__);           \
		if(yzTimed_) ::yz::TimeEnd(strm);                                       \
		::yz::CountLaunches(1);                                                   \
		::yz::Check(cudaGetLastError(), #kernel);                                 \
	} while(0)

void SetLastError(const std::string &m);

//--------------------------------------------------------------------------
//  device buffer (grows, never shrinks; no allocation when large enough)
//--------------------------------------------------------------------------
//  The finest level's stencil: the slices of 32 rows (SELL-32) whose every
//  row has the pattern's most common column set relative to the row (the
//  interior rows of the film: columns i + off[k], ascending) are flagged;
//  their columns are computed, not loaded.  slice null: no flagged slices.
struct Sten
{
	const unsigned char *slice;
	int len;
	int off[16];
};

template<class T>
struct DBuf
{
	T *p = nullptr;
	size_t cap = 0;
	DBuf() = default;
	DBuf(const DBuf &) = delete;
	DBuf &operator=(const DBuf &) = delete;
	~DBuf() { if(p) cudaFree(p); }
	T *get() const { return p; }
	//  a buffer that must grow takes half as much again, so that sizes that
	//  creep up from solve to solve (the coarse levels of the hierarchy) do
	//  not free and allocate (each a device-wide synchronisation) every time
	void reserve(size_t n)
	{
		if(n <= cap) return;
		const size_t grown = cap ? cap + cap / 2 : 0;
		if(p) { cudaFree(p); p = nullptr; cap = 0; }
		size_t want = n < 16 ? 16 : n;
		if(grown > want) want = grown;
		YZ_CUDA(cudaMalloc(&p, want * sizeof(T)));
		cap = want;
	}
	void upload(const T *h, size_t n, cudaStream_t st)
	{
		reserve(n);
		if(n) YZ_CUDA(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
	}
	void download(T *h, size_t n, cudaStream_t st) const
	{
		if(n) YZ_CUDA(cudaMemcpyAsync(h, p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
	}
};

//--------------------------------------------------------------------------
//  the deterministic reduction tree (the oracle's DetSum, yzo_solver.cpp):
//  chunk b of 256 elements per block of 256 threads, thread t holds element
//  b*256 + t, pairwise fold over the block; the chunk sums are summed
//  strided by 256 threads (thread t: chunks t, t+256, ... from 0.0) and
//  folded the same way by the block that finishes last.  One element per
//  thread keeps every SM busy at the sizes of a film (n / 256 blocks).
//--------------------------------------------------------------------------
constexpr int kRT = 256;
constexpr int kRK = 1;
constexpr int kRChunk = kRT * kRK;

inline int RedBlocks(int n) { const int nb = (n + kRChunk - 1) / kRChunk; return nb > 0 ? nb : 1; }

//  Fold Q values per thread over a block of 256 (same order as Tree256).
//  sh: Q*256 doubles of shared memory.  Result valid in thread 0.
template<int Q>
__device__ __forceinline__ void BlockTree(double (&a)[Q], double *sh)
{
	const int t = threadIdx.x;
#pragma unroll
	for(int q = 0; q < Q; ++q) sh[q * kRT + t] = a[q];
	__syncthreads();
#pragma unroll
	for(int off = kRT / 2; off >= 32; off >>= 1)
	{
		if(t < off)
		{
#pragma unroll
			for(int q = 0; q < Q; ++q) sh[q * kRT + t] = sh[q * kRT + t] + sh[q * kRT + t + off];
		}
		__syncthreads();
	}
	if(t < 32)
	{
#pragma unroll
		for(int q = 0; q < Q; ++q)
		{
			double v = sh[q * kRT + t];
#pragma unroll
			for(int off = 16; off >= 1; off >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, off);
			a[q] = v;
		}
	}
}

//  Reduction scratch: Q partial arrays of `blocks` doubles and a counter.
struct RedScratch
{
	double *part;          // [Q][maxBlocks]
	unsigned int *counter; // one per reduction site
	int maxBlocks;
};

//  Called by every block after its threads hold their per-thread sums a[q]:
//  writes the block's partials; the last block to arrive folds them all and
//  returns true with the totals in tot[q] (valid in every thread of it).
template<int Q>
__device__ __forceinline__ bool GridFold(double (&a)[Q], double *sh, const RedScratch rs, double (&tot)[Q])
{
	__shared__ bool amLast;
	BlockTree<Q>(a, sh);
	const int t = threadIdx.x;
	if(t == 0)
	{
#pragma unroll
		for(int q = 0; q < Q; ++q) rs.part[q * rs.maxBlocks + blockIdx.x] = a[q];
		__threadfence();
		const unsigned prev = atomicAdd(rs.counter, 1u);
		amLast = (prev == gridDim.x - 1);
	}
	__syncthreads();
	if(!amLast) return false;
	__threadfence();
	double b[Q];
#pragma unroll
	for(int q = 0; q < Q; ++q)
	{
		double s = 0.0;
		for(int j = t; j < (int)gridDim.x; j += kRT) s = s + __ldcg(&rs.part[q * rs.maxBlocks + j]);
		b[q] = s;
	}
	__syncthreads();
	BlockTree<Q>(b, sh);
	__shared__ double bc[Q];
	if(t == 0)
	{
#pragma unroll
		for(int q = 0; q < Q; ++q) bc[q] = b[q];
		*rs.counter = 0u;
	}
	__syncthreads();
#pragma unroll
	for(int q = 0; q < Q; ++q) tot[q] = bc[q];
	return true;
}

//--------------------------------------------------------------------------
//  exclusive scan of n ints into out[0..n] (out[n] = total); integer, so
//  the order of the additions does not matter.  Scratch: ScanScratchSize(n).
//--------------------------------------------------------------------------
size_t ScanScratchSize(int n);
void ScanExclusive(const int *in, int *out, int n, int *scratch, cudaStream_t st);

//  Grid size for a grid-stride kernel over n items.
inline int GridFor(long long n, int block, int cap = 148 * 16)
{
	long long g = (n + block - 1) / block;
	if(g < 1) g = 1;
	if(g > cap) g = cap;
	return (int)g;
}

} // namespace yz
