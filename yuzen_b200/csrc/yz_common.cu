// yz_common.cu -- launch accounting, the last-error string and the integer scan.
#include "yz_common.cuh"

#include <cstdlib>

#include <mutex>

namespace yz {

std::atomic<long long> g_launches{0};
thread_local long long t_launches = 0;

//  per-launch timing of one kernel (yz_time_kernel)
namespace {
std::mutex g_timeMutex;
std::string g_timeName;                       // read and written under g_timeMutex
std::atomic<bool> g_timeOn{false};            // a name is selected (the launch path's fast test)
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_timePairs;
//  the event that opens a timed launch, per host thread: contexts driven
//  from several threads at once each pair their own events
thread_local cudaEvent_t t_timeOpen = nullptr;
}

bool TimedKernel(const char *name)
{
	if(!g_timeOn.load(std::memory_order_acquire)) return false;
	std::lock_guard<std::mutex> lk(g_timeMutex);
	return !g_timeName.empty() && g_timeName == name;
}

bool PdlOn()
{
	static const char *env = std::getenv("YZ_PDL");
	static const bool on = env && env[0] == '1';
	return on;
}

bool TimingActive() { return g_timeOn.load(std::memory_order_acquire); }

void TimeBegin(cudaStream_t st)
{
	std::lock_guard<std::mutex> lk(g_timeMutex);
	cudaEvent_t e;
	Check(cudaEventCreate(&e), "cudaEventCreate");
	Check(cudaEventRecord(e, st), "cudaEventRecord");
	t_timeOpen = e;
}

void TimeEnd(cudaStream_t st)
{
	std::lock_guard<std::mutex> lk(g_timeMutex);
	cudaEvent_t e;
	Check(cudaEventCreate(&e), "cudaEventCreate");
	Check(cudaEventRecord(e, st), "cudaEventRecord");
	g_timePairs.push_back({t_timeOpen, e});
	t_timeOpen = nullptr;
}

long long TimeCount()
{
	std::lock_guard<std::mutex> lk(g_timeMutex);
	return (long long)g_timePairs.size();
}

void TimeDropLast(long long k)
{
	std::lock_guard<std::mutex> lk(g_timeMutex);
	for(; k > 0 && !g_timePairs.empty(); --k)
	{
		auto &p = g_timePairs.back();
		cudaEventDestroy(p.first);
		cudaEventDestroy(p.second);
		g_timePairs.pop_back();
	}
}

void TimeSelect(const char *name)
{
	std::lock_guard<std::mutex> lk(g_timeMutex);
	for(auto &p : g_timePairs) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
	g_timePairs.clear();
	g_timeName = name ? name : "";
	g_timeOn.store(!g_timeName.empty(), std::memory_order_release);
}

void TimeRead(double *ms, long long *count)
{
	std::lock_guard<std::mutex> lk(g_timeMutex);
	double total = 0;
	for(auto &p : g_timePairs)
	{
		Check(cudaEventSynchronize(p.second), "cudaEventSynchronize");
		float t = 0;
		Check(cudaEventElapsedTime(&t, p.first, p.second), "cudaEventElapsedTime");
		total += t;
	}
	if(ms) *ms = total;
	if(count) *count = (long long)g_timePairs.size();
}

namespace {
thread_local std::string t_lastError;
constexpr int kScanBlock = 1024;

__global__ void ScanBlocks(const int *__restrict__ in, int *__restrict__ out, int n, int *__restrict__ blockSums)
{
	__shared__ int warpSums[kScanBlock / 32];
	const int i = blockIdx.x * kScanBlock + threadIdx.x;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int v = (i < n) ? in[i] : 0;
	//  inclusive scan in the warp
	for(int off = 1; off < 32; off <<= 1)
	{
		const int u = __shfl_up_sync(0xffffffffu, v, off);
		if(lane >= off) v += u;
	}
	if(lane == 31) warpSums[warp] = v;
	__syncthreads();
	if(warp == 0)
	{
		int w = warpSums[lane];
		for(int off = 1; off < 32; off <<= 1)
		{
			const int u = __shfl_up_sync(0xffffffffu, w, off);
			if(lane >= off) w += u;
		}
		warpSums[lane] = w;
	}
	__syncthreads();
	const int incl = v + (warp > 0 ? warpSums[warp - 1] : 0);
	if(i < n) out[i] = incl - ((i < n) ? in[i] : 0);	// exclusive within the block
	if(threadIdx.x == kScanBlock - 1) blockSums[blockIdx.x] = incl;
}

//  one block scans the block sums in tiles of 1024 (exclusive), total at end
__global__ void ScanSums(int *blockSums, int nb, int *total)
{
	__shared__ int warpSums[kScanBlock / 32];
	__shared__ int carry;
	if(threadIdx.x == 0) carry = 0;
	__syncthreads();
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for(int base = 0; base < nb; base += kScanBlock)
	{
		const int i = base + threadIdx.x;
		const int x = (i < nb) ? blockSums[i] : 0;
		int v = x;
		for(int off = 1; off < 32; off <<= 1)
		{
			const int u = __shfl_up_sync(0xffffffffu, v, off);
			if(lane >= off) v += u;
		}
		if(lane == 31) warpSums[warp] = v;
		__syncthreads();
		if(warp == 0)
		{
			int w = warpSums[lane];
			for(int off = 1; off < 32; off <<= 1)
			{
				const int u = __shfl_up_sync(0xffffffffu, w, off);
				if(lane >= off) w += u;
			}
			warpSums[lane] = w;
		}
		__syncthreads();
		const int incl = v + (warp > 0 ? warpSums[warp - 1] : 0);
		const int c = carry;
		if(i < nb) blockSums[i] = c + incl - x;
		__syncthreads();
		if(threadIdx.x == kScanBlock - 1) carry = c + incl;
		__syncthreads();
	}
	if(threadIdx.x == 0) *total = carry;
}

__global__ void ScanAdd(int *out, int n, const int *blockSums, const int *total)
{
	const int i = blockIdx.x * kScanBlock + threadIdx.x;
	if(i < n) out[i] += blockSums[blockIdx.x];
	if(i == 0) out[n] = *total;
}
} // namespace

void SetLastError(const std::string &m) { t_lastError = m; }
const char *LastError() { return t_lastError.c_str(); }

size_t ScanScratchSize(int n) { return (size_t)((n + kScanBlock - 1) / kScanBlock) + 2; }

void ScanExclusive(const int *in, int *out, int n, int *scratch, cudaStream_t st)
{
	const int nb = (n + kScanBlock - 1) / kScanBlock;
	if(n <= 0)
	{
		YZ_CUDA(cudaMemsetAsync(out, 0, sizeof(int), st));
		return;
	}
	int *sums = scratch, *total = scratch + nb;
	YZ_LAUNCH(ScanBlocks, nb, kScanBlock, 0, st, in, out, n, sums);
	YZ_LAUNCH(ScanSums, 1, kScanBlock, 0, st, sums, nb, total);
	YZ_LAUNCH(ScanAdd, nb, kScanBlock, 0, st, out, n, sums, total);
}

} // namespace yz
