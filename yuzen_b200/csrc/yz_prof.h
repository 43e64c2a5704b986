// yz_prof.h -- named parts of a run: NVTX ranges, and device time per name.
//
// The reference labels the parts of its step with YUZEN_PROF("name") scopes
// (util/Profile.h:125-127; h.assemble, h.linsolve, lin.precond, lin.iterate,
// ...): with the environment variable YUZEN_PROFILE set (to anything but 0)
// each scope adds its wall-clock time and one call to the name's total, and
// the totals go to standard error at exit, one line a name:
//
//     [profile] threads 1
//     [profile] h.linsolve        1060      12.345678
//
// The device path keeps the names, the switch and the line format.  What a
// scope measures is the device time of the work it queued on its stream: a
// CUDA event is recorded on the stream where the scope opens and another
// where it closes, and the time between them is added once both have
// completed (the host does not wait for them; completed pairs are summed as
// new scopes close, the rest at exit).  Nested scopes are each inclusive.
// A scope opened while its stream is being captured into a graph times
// nothing (events recorded there would become graph nodes).
//
// Every scope also opens an NVTX range of its name, switch or no switch, so
// a profiler's timeline shows the parts (an NVTX range costs next to nothing
// when no tool is attached).  Nothing here changes what is computed.
#pragma once

#include <cuda_runtime.h>

namespace yz {
namespace prof {

//  YUZEN_PROFILE set and not "0" (read once)
bool Enabled();

class Scope
{
public:
	Scope(const char *name, cudaStream_t st);
	~Scope();
	Scope(const Scope &) = delete;
	Scope &operator=(const Scope &) = delete;

private:
	int _id = -1;
	cudaStream_t _st = nullptr;
	cudaEvent_t _e0 = nullptr;
};

//  the totals so far (every completed pair summed first), in the order the
//  names were first used; false past the last
bool Entry(int index, const char **name, long long *calls, double *seconds);
void Reset();
//  the table to standard error in the reference's format
void Report();

} // namespace prof
} // namespace yz

#define YZ_PROF_CAT2(a, b) a##b
#define YZ_PROF_CAT(a, b) YZ_PROF_CAT2(a, b)
//  times the rest of the enclosing block under the given name, on stream st
#define YZ_PROF(name, st) ::yz::prof::Scope YZ_PROF_CAT(yz_prof_scope_, __LINE__)(name, st)
