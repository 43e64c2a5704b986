/*
 * oracle_backend.cpp -- TEST INFRASTRUCTURE: the linear-solver backend of the
 * CPU oracle binary (the reference's own sources compiled by oracle/Makefile).
 *
 * The reference's LinearSolverBackend.cpp needs Eigen 3.4.0 and AMGCL 1.4.4,
 * neither of which is available, so this file provides the factory
 * MakeLinearSolverBackend (LinearSolverBackend.h:130-131) in its place, with
 * the CPU restatement of both backends from oracle/solver/yzo_solver.cpp:
 *   "amgcl"            -> BiCGStab + SA-AMG(SPAI0)   (AmgclBackend, :539-728)
 *   "eigen"            -> BiCGStab + ILU(0)          (EigenBackend, :272-516)
 *   "auto"             -> amgcl in 2-D, eigen in 1-D (factory, :759-804)
 *   anything else      -> eigen (the reference's rule)
 * With the b200 adapter linked in (YZ_WITH_B200), "b200" creates the GPU
 * backend of yuzen_b200/host/yz_backend_adapter.cpp; since the reference's
 * input reader (compiled unchanged) accepts only auto / eigen / amgcl,
 * YZ_BACKEND=b200 in the environment makes every request for the 2-D AMG
 * backend (amgcl, or auto in 2-D) return it.
 *
 * Dump hook: with YZO_DUMP_DIR set, every solve writes its matrix (storage
 * order and sorted mirror), boundary flags, right-hand side, initial guess and
 * the oracle's answer to YZO_DUMP_DIR/solve_NNNNN.bin (format in
 * tests/golden/dumpio.py). YZO_DUMP_MAX caps the count (default 64).
 */
#include "LinearSolverBackend.h"
#include "CRS_Matrix.h"
#include "YuzenUtil.h"

#include "yzo_solver.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#ifdef YZ_WITH_B200
ILinearSolverBackend* MakeB200LinearSolverBackend();
#endif

namespace {

void DumpSolve(const yzo_settings &s, int flavour, const CRS_Matrix &crs, const double *rhs,
               const double *x0, const double *x, int ret, int iter, double resid)
{
	static const char *dir = std::getenv("YZO_DUMP_DIR");
	if(!dir) return;
	static int count = 0;
	static const int maxCount = std::getenv("YZO_DUMP_MAX") ? std::atoi(std::getenv("YZO_DUMP_MAX")) : 64;
	if(count >= maxCount) return;
	char path[4096];
	std::snprintf(path, sizeof(path), "%s/solve_%05d.bin", dir, count++);
	FILE *f = std::fopen(path, "wb");
	if(!f) return;
	const int n = crs.RowSize(), nnz = crs.NonZero();
	const char magic[8] = {'Y','Z','D','U','M','P','1','\0'};
	std::fwrite(magic, 1, 8, f);
	int hdr[8] = {n, nnz, s.precondition, s.scaling, s.max_iteration, s.conc, flavour, ret};
	std::fwrite(hdr, sizeof(int), 8, f);
	std::fwrite(&iter, sizeof(int), 1, f);
	std::fwrite(&s.epsilon, sizeof(double), 1, f);
	std::fwrite(&resid, sizeof(double), 1, f);
	std::fwrite(crs.RowPtrData(), sizeof(int), (size_t)n + 1, f);
	std::fwrite(crs.ColIndData(), sizeof(int), (size_t)nnz, f);
	std::fwrite(crs.SortedColIndData(), sizeof(int), (size_t)nnz, f);
	std::fwrite(crs.SortedSrcData(), sizeof(int), (size_t)nnz, f);
	std::vector<int> bc((size_t)n);
	for(int i = 0; i < n; ++i) bc[(size_t)i] = crs.IsBC(i) ? 1 : 0;
	std::fwrite(bc.data(), sizeof(int), (size_t)n, f);
	std::fwrite(crs.ValuesData(), sizeof(double), (size_t)nnz, f);
	std::fwrite(rhs, sizeof(double), (size_t)n, f);
	std::fwrite(x0, sizeof(double), (size_t)n, f);
	std::fwrite(x, sizeof(double), (size_t)n, f);
	std::fclose(f);
}

class OracleBackend : public ILinearSolverBackend
{
public:
	OracleBackend(int flavour, const char *name) : _flavour(flavour), _name(name), _s(yzo_create(flavour)) {}
	virtual ~OracleBackend() { yzo_destroy(_s); }
	virtual const char* Name() const { return _name; }
	virtual void Build(int, int, int, int) {}

	virtual int Solve(const LinearSolverSettings &ls, CRS_Matrix &crs,
	                  Vector<double> &rhs, Vector<double> &x, int &iter, double &resid)
	{
		yzo_settings s;
		s.precondition = (int)ls.precondition;
		s.scaling = ls.scaling ? 1 : 0;
		s.max_iteration = ls.maxIteration;
		s.epsilon = ls.epsilon;
		s.conc = ls.conc ? 1 : 0;
		const int n = crs.RowSize();
		std::vector<double> x0;
		const bool dump = std::getenv("YZO_DUMP_DIR") != 0;
		if(dump) x0.assign(x.data(), x.data() + n);
		const int ret = yzo_solve(_s, &s, n, crs.RowPtrData(), crs.SortedColIndData(), crs.SortedSrcData(),
		                          crs.ValuesData(), rhs.data(), x.data(), &iter, &resid);
		if(dump) DumpSolve(s, _flavour, crs, rhs.data(), x0.data(), x.data(), ret, iter, resid);
		return ret;
	}

	virtual std::vector<double> Memory() const
	{
		double m[8];
		const int k = yzo_memory(_s, m, 8);
		return std::vector<double>(m, m + k);
	}
	virtual void SetMemory(const std::vector<double> &m)
	{
		yzo_set_memory(_s, m.data(), (int)m.size());
	}

private:
	int _flavour;
	const char *_name;
	yzo_solver *_s;
};

} // namespace

ILinearSolverBackend* MakeLinearSolverBackend(const std::string &name, int inPlane)
{
#ifdef YZ_WITH_B200
	if(name == "b200") return MakeB200LinearSolverBackend();
	if(const char *e = std::getenv("YZ_BACKEND"))
		if(std::string(e) == "b200" && (name == "amgcl" || (name == "auto" && inPlane >= 2)))
			return MakeB200LinearSolverBackend();
#endif
	if(name == "auto")
	{
		if(inPlane >= 2) return new OracleBackend(YZO_AMG, "amgcl");
		return new OracleBackend(YZO_ILU0, "eigen");
	}
	if(name == "amgcl") return new OracleBackend(YZO_AMG, "amgcl");
	return new OracleBackend(YZO_ILU0, "eigen");
}
