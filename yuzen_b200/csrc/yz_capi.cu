// yz_capi.cu -- the extern "C" entry points of include/yuzen_b200.h.
// Every call catches what the C++ side throws and turns it into a status.
#include "yz_solver_impl.h"
#include "yz_step_impl.h"

#include <cstring>

struct yz_solver
{
	std::unique_ptr<yz::Solver> s;
};

struct yz_step
{
	std::unique_ptr<yz::Step> s;
};

namespace {
template<class F> int Guard(F &&f)
{
	try { return f(); }
	catch(const yz::UsageError &e) { yz::SetLastError(e.what()); return -1; }
	catch(const yz::StepFailed &e) { yz::SetLastError(e.what()); return -3; }
	catch(const yz::CudaError &e) { yz::SetLastError(e.what()); return -2; }
	catch(const std::exception &e) { yz::SetLastError(e.what()); return -2; }
	catch(...) { yz::SetLastError("unknown error"); return -2; }
}
}

extern "C" {

const char *yz_last_error(void) { return yz::LastError(); }

int yz_solver_create(int device, yz_solver **out)
{
	return Guard([&] {
		if(!out) throw yz::UsageError("yz_solver_create: out is null");
		int count = 0;
		yz::Check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
		if(device < 0 || device >= count) throw yz::UsageError("yz_solver_create: no such CUDA device");
		yz_solver *h = new yz_solver();
		h->s.reset(new yz::Solver(device));
		*out = h;
		return 0;
	});
}

int yz_solver_destroy(yz_solver *s)
{
	return Guard([&] { delete s; return 0; });
}

int yz_solver_set_pattern(yz_solver *s, int n, int nnz, const int *rowptr, const int *scol, const int *ssrc)
{
	return Guard([&] {
		if(!s || !rowptr || !scol || !ssrc) throw yz::UsageError("yz_solver_set_pattern: null argument");
		s->s->SetPattern(n, nnz, rowptr, scol, ssrc);
		return 0;
	});
}

int yz_solver_solve(yz_solver *s, const yz_settings *set, const double *values, const double *rhs, double *x,
                    int *iter, double *resid)
{
	return Guard([&] {
		if(!s || !set || !values || !rhs || !x || !iter || !resid) throw yz::UsageError("yz_solver_solve: null argument");
		return s->s->SolveHost(*set, values, rhs, x, *iter, *resid);
	});
}

int yz_solver_solve_device(yz_solver *s, const yz_settings *set, const double *dv, const double *dr, double *dx,
                           int *iter, double *resid)
{
	return Guard([&] {
		if(!s || !set || !dv || !dr || !dx || !iter || !resid) throw yz::UsageError("yz_solver_solve_device: null argument");
		return s->s->Solve(*set, dv, dr, dx, *iter, *resid);
	});
}

int yz_solver_set_precision(yz_solver *s, int precision)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_set_precision: null solver");
		s->s->SetPrecision(precision);
		return 0;
	});
}

int yz_solver_set_amg_reuse(yz_solver *s, int maxSolves)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_set_amg_reuse: null solver");
		s->s->SetAmgReuse(maxSolves);
		return 0;
	});
}

int yz_solver_set_graph_loop(yz_solver *s, int on)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_set_graph_loop: null solver");
		s->s->SetGraphLoop(on != 0);
		return 0;
	});
}

int yz_solver_memory(const yz_solver *s, double *out, int cap)
{
	return Guard([&] {
		if(!s || (!out && cap > 0)) throw yz::UsageError("yz_solver_memory: null argument");
		const std::vector<double> m = s->s->Memory();
		for(int i = 0; i < (int)m.size() && i < cap; ++i) out[i] = m[(size_t)i];
		return (int)m.size();
	});
}

int yz_solver_set_memory(yz_solver *s, const double *m, int len)
{
	return Guard([&] {
		if(!s || (!m && len > 0)) throw yz::UsageError("yz_solver_set_memory: null argument");
		s->s->SetMemory(m, len);
		return 0;
	});
}

int yz_solver_levels(const yz_solver *s)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_levels: null solver");
		return s->s->LevelCount();
	});
}

int yz_solver_level_info(const yz_solver *s, int level, int *rows, int *nnz_a, int *nnz_p, int *direct)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_level_info: null solver");
		s->s->LevelInfo(level, rows, nnz_a, nnz_p, direct);
		return 0;
	});
}

int yz_solver_level_copy(const yz_solver *s, int level, int *a_ptr, int *a_col, double *a_val, int *p_ptr, int *p_col,
                         double *p_val, int *agg)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_level_copy: null solver");
		const_cast<yz_solver *>(s)->s->LevelCopy(level, a_ptr, a_col, a_val, p_ptr, p_col, p_val, agg);
		return 0;
	});
}

int yz_solver_last_timing(const yz_solver *s, double *setup_ms, double *iterate_ms)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_last_timing: null solver");
		s->s->Timing(setup_ms, iterate_ms);
		return 0;
	});
}

long long yz_solver_launches(const yz_solver *s) { return s ? s->s->Launches() : -1; }

long long yz_launch_count(void) { return yz::g_launches.load(); }

int yz_dot_noalloc(int n, const double *d_x, const double *d_y, double *d_out, void *stream)
{
	return Guard([&] {
		yz::DotNoAlloc(n, d_x, d_y, d_out, static_cast<cudaStream_t>(stream));
		return 0;
	});
}

long long yz_dot_noalloc_max(void) { return yz::NoAllocMaxElements(); }

int yz_time_kernel(const char *name)
{
	return Guard([&] { yz::TimeSelect(name); return 0; });
}

int yz_kernel_time(double *total_ms, long long *launches)
{
	return Guard([&] { yz::TimeRead(total_ms, launches); return 0; });
}

int yz_dot(int n, const double *x, const double *y, double *out)
{
	return Guard([&] {
		if(n < 0 || (n > 0 && (!x || !y)) || !out) throw yz::UsageError("yz_dot: bad argument");
		*out = yz::DeviceDot(n, x, y);
		return 0;
	});
}

int yz_spmv(int n, int nnz, const int *rowptr, const int *col, const double *val, const double *x, double *y)
{
	return Guard([&] {
		if(n <= 0 || nnz < 0 || !rowptr || !col || !val || !x || !y) throw yz::UsageError("yz_spmv: bad argument");
		yz::DeviceSpmv(n, nnz, rowptr, col, val, x, y);
		return 0;
	});
}

//--------------------------------------------------------------------------
//  the whole step
//--------------------------------------------------------------------------
int yz_step_create(int device, const yz_step_params *p, const double *h, const double *c, const double *s, yz_step **out)
{
	return Guard([&] {
		if(!p || !h || !c || !s || !out) throw yz::UsageError("yz_step_create: null argument");
		int count = 0;
		yz::Check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
		if(device < 0 || device >= count) throw yz::UsageError("yz_step_create: no such CUDA device");
		yz_step *st = new yz_step();
		try { st->s.reset(new yz::Step(device, *p, h, c, s)); }
		catch(...) { delete st; throw; }
		*out = st;
		return 0;
	});
}

int yz_step_destroy(yz_step *st)
{
	return Guard([&] { delete st; return 0; });
}

int yz_step_set_precision(yz_step *st, int precision)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_precision: null step");
		st->s->SetPrecision(precision);
		return 0;
	});
}

int yz_step_set_amg_reuse(yz_step *st, int maxSolves)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_amg_reuse: null step");
		st->s->SetAmgReuse(maxSolves);
		return 0;
	});
}

int yz_step_set_graph_loop(yz_step *st, int on)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_graph_loop: null step");
		st->s->SetGraphLoop(on != 0);
		return 0;
	});
}

int yz_step_set_energy(yz_step *st, int on)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_energy: null step");
		st->s->SetEnergy(on != 0);
		return 0;
	});
}

int yz_step_energy(yz_step *st, double *F, double *D)
{
	return Guard([&] {
		if(!st || !F || !D) throw yz::UsageError("yz_step_energy: null argument");
		st->s->Energy(*F, *D);
		return 0;
	});
}

int yz_step_advance(yz_step *st, int nsteps, yz_step_stats *stats)
{
	return Guard([&] {
		if(!st || nsteps < 0) throw yz::UsageError("yz_step_advance: bad argument");
		yz_step_stats local;
		std::memset(&local, 0, sizeof local);
		st->s->Advance(nsteps, local);
		if(stats) *stats = local;
		return 0;
	});
}

int yz_step_get_fields(yz_step *st, double *h, double *c)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_get_fields: null step");
		st->s->GetFields(h, c);
		return 0;
	});
}

int yz_step_set_fields(yz_step *st, const double *h, const double *c)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_fields: null step");
		st->s->SetFields(h, c);
		return 0;
	});
}

int yz_step_pattern(yz_step *st, int *rowptr, int *col, int *bc)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_pattern: null step");
		return st->s->Pattern(rowptr, col, bc);
	});
}

int yz_step_system(yz_step *st, const double *h_old, const double *h, double dt, double *ia, double *rhs)
{
	return Guard([&] {
		if(!st || !h_old || !h || !ia || !rhs) throw yz::UsageError("yz_step_system: null argument");
		st->s->System(h_old, h, dt, ia, rhs);
		return 0;
	});
}

int yz_step_conc_pattern(yz_step *st, int *rowptr, int *col)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_conc_pattern: null step");
		return st->s->ConcPattern(rowptr, col);
	});
}

int yz_step_conc_system(yz_step *st, const double *h, const double *c, double dt, double *values, double *rhs)
{
	return Guard([&] {
		if(!st || !h || !c || !values || !rhs) throw yz::UsageError("yz_step_conc_system: null argument");
		st->s->ConcSystem(h, c, dt, values, rhs);
		return 0;
	});
}

int yz_pattern_2d(const yz_step_params *p, int *rowptr, int *col, int *bc)
{
	return Guard([&] {
		if(!p) throw yz::UsageError("yz_pattern_2d: null params");
		yz::CheckParams(*p);
		std::vector<int> rp, cl, isbc, ghost, partner;
		yz::BuildPattern2D(*p, rp, cl, isbc, ghost, partner);
		if(rowptr) std::copy(rp.begin(), rp.end(), rowptr);
		if(col) std::copy(cl.begin(), cl.end(), col);
		if(bc) std::copy(isbc.begin(), isbc.end(), bc);
		return (int)cl.size();
	});
}

} // extern "C"
