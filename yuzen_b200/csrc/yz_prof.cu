// yz_prof.cu -- the named scopes of yz_prof.h: NVTX ranges and, with
// YUZEN_PROFILE set, device time per name from event pairs.
#include "yz_prof.h"

#include <nvtx3/nvToolsExt.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace yz {
namespace prof {
namespace {

struct Total
{
	std::string name;
	long long calls = 0;
	double seconds = 0.0;
};

struct Pending
{
	int id;
	int device;
	cudaEvent_t e0, e1;
};

//  pairs waiting for their events beyond this many are waited for
constexpr size_t kMaxPending = 4096;

std::mutex g_mutex;
std::vector<Total> g_totals;
std::deque<Pending> g_pending;
std::map<int, std::vector<cudaEvent_t>> g_pool;   // free events by device

int IdOf(const char *name)
{
	for(size_t i = 0; i < g_totals.size(); ++i)
		if(g_totals[i].name == name) return (int)i;
	g_totals.push_back(Total{name, 0, 0.0});
	return (int)g_totals.size() - 1;
}

cudaEvent_t TakeEvent(int device)
{
	std::vector<cudaEvent_t> &v = g_pool[device];
	if(!v.empty())
	{
		cudaEvent_t e = v.back();
		v.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	if(cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
	return e;
}

//  adds the pair's time (false: not complete yet, and wait is false)
bool Settle(const Pending &p, bool wait)
{
	int cur = 0;
	cudaGetDevice(&cur);
	if(cur != p.device) cudaSetDevice(p.device);
	cudaError_t q = wait ? cudaEventSynchronize(p.e1) : cudaEventQuery(p.e1);
	if(q == cudaErrorNotReady) { if(cur != p.device) cudaSetDevice(cur); return false; }
	float ms = 0.0f;
	if(q == cudaSuccess && cudaEventElapsedTime(&ms, p.e0, p.e1) == cudaSuccess)
	{
		g_totals[(size_t)p.id].seconds += 1e-3 * (double)ms;
		++g_totals[(size_t)p.id].calls;
	}
	else cudaGetLastError();
	g_pool[p.device].push_back(p.e0);
	g_pool[p.device].push_back(p.e1);
	if(cur != p.device) cudaSetDevice(cur);
	return true;
}

//  sums every completed pair (all of them when wait)
void Drain(bool wait)
{
	for(auto it = g_pending.begin(); it != g_pending.end();)
	{
		if(Settle(*it, wait)) it = g_pending.erase(it);
		else ++it;
	}
	while(g_pending.size() > kMaxPending)
	{
		Settle(g_pending.front(), true);
		g_pending.pop_front();
	}
}

} // namespace

bool Enabled()
{
	static const bool on = []() {
		const char *e = std::getenv("YUZEN_PROFILE");
		const bool b = (e != nullptr && *e != 0 && std::strcmp(e, "0") != 0);
		if(b) std::atexit(Report);
		return b;
	}();
	return on;
}

Scope::Scope(const char *name, cudaStream_t st)
{
	nvtxRangePushA(name);
	if(!Enabled()) return;
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	if(cudaStreamIsCapturing(st, &cs) != cudaSuccess) { cudaGetLastError(); return; }
	if(cs != cudaStreamCaptureStatusNone) return;
	int device = 0;
	if(cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return; }
	std::lock_guard<std::mutex> lk(g_mutex);
	cudaEvent_t e = TakeEvent(device);
	if(!e) return;
	if(cudaEventRecord(e, st) != cudaSuccess) { cudaGetLastError(); g_pool[device].push_back(e); return; }
	_id = IdOf(name);
	_st = st;
	_e0 = e;
}

Scope::~Scope()
{
	if(_e0)
	{
		int device = 0;
		cudaGetDevice(&device);
		std::lock_guard<std::mutex> lk(g_mutex);
		cudaEvent_t e1 = TakeEvent(device);
		if(e1 && cudaEventRecord(e1, _st) == cudaSuccess)
		{
			g_pending.push_back(Pending{_id, device, _e0, e1});
			Drain(false);
		}
		else
		{
			cudaGetLastError();
			g_pool[device].push_back(_e0);
			if(e1) g_pool[device].push_back(e1);
		}
	}
	nvtxRangePop();
}

bool Entry(int index, const char **name, long long *calls, double *seconds)
{
	std::lock_guard<std::mutex> lk(g_mutex);
	Drain(true);
	if(index < 0 || index >= (int)g_totals.size()) return false;
	const Total &t = g_totals[(size_t)index];
	if(name) *name = t.name.c_str();
	if(calls) *calls = t.calls;
	if(seconds) *seconds = t.seconds;
	return true;
}

void Reset()
{
	std::lock_guard<std::mutex> lk(g_mutex);
	Drain(true);
	for(Total &t : g_totals) { t.calls = 0; t.seconds = 0.0; }
}

void Report()
{
	std::lock_guard<std::mutex> lk(g_mutex);
	Drain(true);
	//  one host thread queues the device's work
	std::fprintf(stderr, "[profile] threads 1\n");
	for(const Total &t : g_totals)
		std::fprintf(stderr, "[profile] %-20s %12lld %14.6f\n", t.name.c_str(), t.calls, t.seconds);
}

} // namespace prof
} // namespace yz
