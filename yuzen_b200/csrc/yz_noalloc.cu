// yz_noalloc.cu -- the deterministic dot product without any allocation.
//
// Some callers cannot allocate device memory: a host code that manages the
// whole device memory itself (and forbids allocations behind its back), a
// code path that must not take the device-wide synchronisation cudaMalloc
// implies, or a caller that hands over only the buffers it already owns.
// For them yz_dot_noalloc computes the same dot product as yz_dot (the
// reduction tree of every BiCGStab dot product, yz_common.cuh), on device
// arrays the caller passes, with its block partials and its counter in one
// static array of this file instead of an allocation.
//
// The array lives as long as the library is loaded, on every device that
// loads it (kScratchDoubles doubles, 512 KiB + 256 B).  Every call shares it
// and it keeps the last call's contents: calls that overlap on the GPU (two
// streams, two host threads) race on it.  The counter that must start at
// zero is cleared by each call before its kernel.  The device address of the
// array is taken once per device, on the first call made with that device
// current, by cudaGetSymbolAddress; that first call should come before any
// stream capture.  The address is kept per device index for the life of the
// process and belongs to the device's primary context: after cudaDeviceReset,
// or under a non-primary driver context, it is stale.
#include "yz_common.cuh"

#include <array>
#include <mutex>

namespace yz {
namespace {

//  block partials the scratch holds; n may be up to that many reduction
//  chunks (kMaxBlocks * kRChunk elements)
constexpr int kMaxBlocks = 65536;
//  the counter in the first 256 bytes, the partials after them
constexpr int kCounterDoubles = 32;
constexpr int kScratchDoubles = kCounterDoubles + kMaxBlocks;

static __device__ __align__(256) double g_noallocScratch[kScratchDoubles];

std::mutex g_addrMutex;
std::array<double *, 128> g_addr{};

double *ScratchAddress(int device)
{
	std::lock_guard<std::mutex> lk(g_addrMutex);
	if(device < 0 || device >= (int)g_addr.size()) throw UsageError("yz_dot_noalloc: device index out of range");
	if(!g_addr[(size_t)device])
	{
		double *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noallocScratch);
		if(e != cudaSuccess) throw CudaError(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
		g_addr[(size_t)device] = p;
	}
	return g_addr[(size_t)device];
}

__global__ void KDotNoAlloc(int n, const double *__restrict__ x, const double *__restrict__ y, RedScratch rs,
                            double *out)
{
	__shared__ double sh[kRT];
	double a[1] = {0.0};
	for(int kk = 0, i = blockIdx.x * kRChunk + threadIdx.x; kk < kRK; ++kk, i += kRT)
	{
		if(i >= n) break;
		a[0] = a[0] + x[i] * y[i];
	}
	double tot[1];
	if(GridFold<1>(a, sh, rs, tot) && threadIdx.x == 0) *out = tot[0];
}

} // namespace

long long NoAllocMaxElements() { return (long long)kMaxBlocks * kRChunk; }

void DotNoAlloc(int n, const double *dx, const double *dy, double *dout, cudaStream_t st)
{
	if(n < 0) throw UsageError("yz_dot_noalloc: n must be >= 0");
	if((long long)n > NoAllocMaxElements())
		throw UsageError("yz_dot_noalloc: n exceeds the maximum of " + std::to_string(NoAllocMaxElements()) +
		                 " elements its static scratch holds");
	if((n > 0 && (!dx || !dy)) || !dout) throw UsageError("yz_dot_noalloc: null pointer");
	int device = 0;
	YZ_CUDA(cudaGetDevice(&device));
	double *scratch = ScratchAddress(device);
	RedScratch rs;
	rs.counter = reinterpret_cast<unsigned int *>(scratch);
	rs.part = scratch + kCounterDoubles;
	rs.maxBlocks = kMaxBlocks;
	YZ_CUDA(cudaMemsetAsync(rs.counter, 0, sizeof(unsigned int), st));
	YZ_LAUNCH(KDotNoAlloc, RedBlocks(n), kRT, 0, st, n, dx, dy, rs, dout);
}

} // namespace yz
