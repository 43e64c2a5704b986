// yz_capi.cu -- the extern "C" entry points of include/yuzen_b200.h.
// Every call catches what the C++ side throws and turns it into a status.
#include "yz_solver_impl.h"
#include "yz_step_impl.h"
#include "yz_cz.h"
#include "yz_prof.h"

#include <cstring>

struct yz_solver
{
	std::unique_ptr<yz::Solver> s;
};

struct yz_step
{
	std::unique_ptr<yz::Step> s;
};

struct yz_cz
{
	std::unique_ptr<yz::CzStep> z;
};

struct yz_unet
{
	std::unique_ptr<yz::Learned> u;
};

namespace yz {
void Conv3x3Host(int H, int W, int cin, int n, int realW, int realH, int relu, const float *x, const float *w,
                 const float *bias, float *y);
}

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

int yz_solver_set_tuning(yz_solver *s, int fuse_from, int coarse_lanes, int fine_sweeps)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_set_tuning: null solver");
		s->s->SetTuning(fuse_from, coarse_lanes, fine_sweeps);
		return 0;
	});
}

int yz_step_set_tuning(yz_step *st, int fuse_from, int coarse_lanes, int fine_sweeps)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_tuning: null step");
		st->s->SetTuning(fuse_from, coarse_lanes, fine_sweeps);
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

long long yz_step_state_size(const yz_step *st) { return st ? (long long)st->s->StateSize() : -1; }

int yz_step_get_state(yz_step *st, double *out)
{
	return Guard([&] {
		if(!st || !out) throw yz::UsageError("yz_step_get_state: null argument");
		st->s->GetState(out);
		return 0;
	});
}

int yz_step_set_state(yz_step *st, const double *in, long long len)
{
	return Guard([&] {
		if(!st || !in || len <= 0) throw yz::UsageError("yz_step_set_state: null argument");
		st->s->SetState(in, (size_t)len);
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

//--------------------------------------------------------------------------
//  the learned preconditioner
//--------------------------------------------------------------------------
int yz_unet_create(int device, int nx, int ny, int capacity, unsigned seed, int activation, yz_unet **out)
{
	return Guard([&] {
		if(!out) throw yz::UsageError("yz_unet_create: out is null");
		int count = 0;
		yz::Check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
		if(device < 0 || device >= count) throw yz::UsageError("yz_unet_create: no such CUDA device");
		yz_unet *h = new yz_unet();
		if(activation != 0 && activation != 1) throw yz::UsageError("yz_unet_create: activation must be 0 or 1");
		try { h->u.reset(new yz::Learned(device, nx, ny, capacity, seed, activation)); }
		catch(...) { delete h; throw; }
		*out = h;
		return 0;
	});
}

int yz_unet_destroy(yz_unet *u)
{
	return Guard([&] { delete u; return 0; });
}

long long yz_unet_param_count(const yz_unet *u) { return u ? (long long)u->u->ParamCount() : -1; }

int yz_unet_get_params(yz_unet *u, float *out)
{
	return Guard([&] {
		if(!u || !out) throw yz::UsageError("yz_unet_get_params: null argument");
		u->u->GetParams(out, 0);
		return 0;
	});
}

int yz_unet_set_params(yz_unet *u, const float *in)
{
	return Guard([&] {
		if(!u || !in) throw yz::UsageError("yz_unet_set_params: null argument");
		u->u->SetParams(in, 0);
		return 0;
	});
}

int yz_unet_forward(yz_unet *u, const float *feat3, float *out)
{
	return Guard([&] {
		if(!u || !feat3 || !out) throw yz::UsageError("yz_unet_forward: null argument");
		u->u->Forward(feat3, out, 0);
		return 0;
	});
}

int yz_unet_loss_grad(yz_unet *u, const float *feat3, const float *target, double *loss, float *grad)
{
	return Guard([&] {
		if(!u || !feat3 || !target || !grad) throw yz::UsageError("yz_unet_loss_grad: null argument");
		const double l = u->u->LossGrad(feat3, target, grad, 0);
		if(loss) *loss = l;
		return 0;
	});
}

int yz_unet_add_sample(yz_unet *u, const double *r, const double *z, const double *diag, const double *h)
{
	return Guard([&] {
		if(!u || !r || !z || !diag) throw yz::UsageError("yz_unet_add_sample: null argument");
		u->u->AddSampleHost(r, z, diag, h, 0);
		return 0;
	});
}

int yz_unet_samples(const yz_unet *u) { return u ? u->u->Samples() : -1; }

int yz_unet_get_sample(yz_unet *u, int k, float *out, int *valid)
{
	return Guard([&] {
		if(!u || !out) throw yz::UsageError("yz_unet_get_sample: null argument");
		const bool v = u->u->GetSample(k, out, 0);
		if(valid) *valid = v ? 1 : 0;
		return 0;
	});
}

int yz_unet_train(yz_unet *u, int iters, int batch, float lr, int holdout, double *loss, double *val_err)
{
	return Guard([&] {
		if(!u) throw yz::UsageError("yz_unet_train: null network");
		if(iters < 0 || batch < 1 || !(lr > 0) || holdout < 0)
			throw yz::UsageError("yz_unet_train: iters >= 0, batch >= 1, lr > 0, holdout >= 0");
		double v = -1.0;
		const double l = u->u->Train(iters, batch, lr, holdout, &v, 0);
		if(loss) *loss = l;
		if(val_err) *val_err = v;
		return 0;
	});
}

int yz_unet_apply(yz_unet *u, const double *d_values, const int *d_rowptr, const double *d_h, const double *d_r,
                  double *d_z, void *stream)
{
	return Guard([&] {
		if(!u || !d_values || !d_rowptr || !d_r || !d_z) throw yz::UsageError("yz_unet_apply: null argument");
		cudaStream_t st = static_cast<cudaStream_t>(stream);
		u->u->SetAux(d_values, d_rowptr, d_h, st);
		u->u->Apply(d_r, d_z, st, nullptr);
		return 0;
	});
}

int yz_solver_set_learned(yz_solver *s, yz_unet *u, int mode, int collect_solves, int per_solve, double cap_factor)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_set_learned: null solver");
		if(mode == 2 && u && !u->u->Trained()) throw yz::UsageError("yz_solver_set_learned: the network is not trained");
		s->s->SetLearned(u ? u->u.get() : nullptr, mode, collect_solves, per_solve, cap_factor);
		return 0;
	});
}

int yz_solver_set_aux(yz_solver *s, const double *d_h)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_set_aux: null solver");
		s->s->SetAux(d_h);
		return 0;
	});
}

int yz_solver_learned_stats(const yz_solver *s, int *solves, int *fallbacks, int *iterations, int *skipped)
{
	return Guard([&] {
		if(!s) throw yz::UsageError("yz_solver_learned_stats: null solver");
		const yz::Solver::LearnedStats &l = s->s->LStats();
		if(solves) *solves = l.solves;
		if(fallbacks) *fallbacks = l.fallbacks;
		if(iterations) *iterations = l.iterations;
		if(skipped) *skipped = l.skipped;
		return 0;
	});
}

int yz_step_set_learned(yz_step *st, const yz_learned_cfg *cfg)
{
	return Guard([&] {
		if(!st) throw yz::UsageError("yz_step_set_learned: null step");
		st->s->SetLearned(cfg);
		return 0;
	});
}

int yz_fault_inject(long long at, long long count)
{
	return Guard([&] {
		if(at < 0 || count < 0) throw yz::UsageError("yz_fault_inject: at and count must be >= 0");
		yz::FaultInject((long)at, (long)count);
		return 0;
	});
}

int yz_profile_enabled(void) { return yz::prof::Enabled() ? 1 : 0; }

int yz_profile_entry(int index, const char **name, long long *calls, double *seconds)
{
	return Guard([&] { return yz::prof::Entry(index, name, calls, seconds) ? 0 : 1; });
}

int yz_profile_reset(void)
{
	return Guard([&] {
		yz::prof::Reset();
		return 0;
	});
}

int yz_conv3x3(int H, int W, int cin, int n, int real_w, int real_h, int relu, const float *x, const float *w,
               const float *bias, float *y)
{
	return Guard([&] {
		if(!x || !w || !y) throw yz::UsageError("yz_conv3x3: null argument");
		yz::Conv3x3Host(H, W, cin, n, real_w, real_h, relu, x, w, bias, y);
		return 0;
	});
}

} // extern "C"

//--------------------------------------------------------------------------
//  seam 3: the ConcZ model's step
//--------------------------------------------------------------------------
int yz_cz_create(int device, const yz_cz_params *p, const double *xc, const double *xf, const double *yc,
                 const double *yf, const double *h, const double *s, const double *c, yz_cz **out)
{
	return Guard([&] {
		if(!p || !xc || !xf || !yc || !yf || !h || !s || !c || !out) throw yz::UsageError("yz_cz_create: null argument");
		yz::CheckCzParams(*p);
		int count = 0;
		yz::Check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
		if(device < 0 || device >= count) throw yz::UsageError("yz_cz_create: no such CUDA device");
		yz_cz *z = new yz_cz();
		try { z->z.reset(new yz::CzStep(device, *p, xc, xf, yc, yf, h, s, c)); }
		catch(...) { delete z; throw; }
		*out = z;
		return 0;
	});
}

int yz_cz_destroy(yz_cz *z)
{
	return Guard([&] { delete z; return 0; });
}

int yz_cz_advance(yz_cz *z, int nsteps, yz_cz_stats *stats)
{
	return Guard([&] {
		if(!z || !stats) throw yz::UsageError("yz_cz_advance: null argument");
		if(nsteps < 0) throw yz::UsageError("yz_cz_advance: nsteps must be >= 0");
		z->z->Advance(nsteps, *stats);
		return 0;
	});
}

int yz_cz_get_fields(yz_cz *z, double *h, double *c)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_get_fields: null model");
		z->z->GetFields(h, c);
		return 0;
	});
}

int yz_cz_set_fields(yz_cz *z, const double *h, const double *c)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_set_fields: null model");
		z->z->SetFields(h, c);
		return 0;
	});
}

int yz_cz_set_precision(yz_cz *z, int precision)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_set_precision: null model");
		z->z->SetPrecision(precision);
		return 0;
	});
}

int yz_cz_set_tuning(yz_cz *z, int fuse_from, int coarse_lanes, int fine_sweeps)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_set_tuning: null model");
		z->z->SetTuning(fuse_from, coarse_lanes, fine_sweeps);
		return 0;
	});
}

int yz_cz_set_learned(yz_cz *z, const yz_learned_cfg *cfg)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_set_learned: null model");
		z->z->SetLearned(cfg);
		return 0;
	});
}

int yz_cz_set_amg_reuse(yz_cz *z, int max_solves)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_set_amg_reuse: null model");
		z->z->SetAmgReuse(max_solves);
		return 0;
	});
}

int yz_cz_parts(yz_cz *z)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_parts: null model");
		z->z->Parts();
		return 0;
	});
}

long long yz_cz_read(yz_cz *z, const char *name, double *out, long long cap)
{
	long long n = -1;
	const int r = Guard([&] {
		if(!z || !name) throw yz::UsageError("yz_cz_read: null argument");
		n = z->z->Read(name, out, cap);
		return 0;
	});
	return r != 0 ? r : n;
}

int yz_cz_pattern(yz_cz *z, int which, int *rowptr, int *col, int *bc)
{
	return Guard([&] {
		if(!z) throw yz::UsageError("yz_cz_pattern: null model");
		return z->z->Pattern(which, rowptr, col, bc);
	});
}

int yz_cz_build_pattern(const yz_cz_params *p, int which, int *rowptr, int *col, int *bc)
{
	return Guard([&] {
		if(!p) throw yz::UsageError("yz_cz_build_pattern: null params");
		yz::CheckCzParams(*p);
		std::vector<int> rh, ch, bh, rc, cc, bcc;
		yz::BuildCzPatterns(*p, rh, ch, bh, rc, cc, bcc);
		const std::vector<int> &R = which ? rc : rh, &C = which ? cc : ch, &B = which ? bcc : bh;
		if(rowptr) std::memcpy(rowptr, R.data(), R.size() * sizeof(int));
		if(col) std::memcpy(col, C.data(), C.size() * sizeof(int));
		if(bc) std::memcpy(bc, B.data(), B.size() * sizeof(int));
		return (int)C.size();
	});
}

int yz_exp_cr(long long n, const double *x, double *y)
{
	return Guard([&] {
		if(n < 0 || (n > 0 && (!x || !y))) throw yz::UsageError("yz_exp_cr: bad argument");
		yz::ExpCrHost(n, x, y);
		return 0;
	});
}
