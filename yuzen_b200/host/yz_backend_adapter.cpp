/*
 * yz_backend_adapter.cpp -- the class a maintainer of the reference adds to
 * drop the B200 linear solve in behind its solver seam.
 *
 * It implements the reference's ILinearSolverBackend
 * (yuzen/src/numerics/LinearSolverBackend.h:56-103) by forwarding to the C ABI
 * of include/yuzen_b200.h.  It is compiled against the reference's headers
 * (CRS_Matrix, Vector, LinearSolverSettings) and linked with
 * libyuzen_b200.so; the factory MakeLinearSolverBackend
 * (LinearSolverBackend.cpp:759-804) returns it for the name "b200":
 *
 *     if(name == "b200") return MakeB200LinearSolverBackend();
 *
 * oracle/Makefile builds the reference's driver with it (target b200) for
 * the drop-in test.
 */
#include "LinearSolverBackend.h"
#include "CRS_Matrix.h"

#include "yuzen_b200.h"

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

class B200Backend : public ILinearSolverBackend
{
public:
	B200Backend() : _s(nullptr), _n(-1), _nnz(-1)
	{
		const char *dev = std::getenv("YZ_DEVICE");
		if(yz_solver_create(dev ? std::atoi(dev) : 0, &_s) != 0)
			throw std::runtime_error(std::string("b200 backend: ") + yz_last_error());
	}
	virtual ~B200Backend() { yz_solver_destroy(_s); }

	virtual const char* Name() const { return "b200"; }

	//  the pattern is handed over with the first solve: it is fixed after
	//  the first assembly (LinearSolverBackend.cpp:301-315)
	virtual void Build(int nRow, int nonZero, int, int) { (void)nRow; (void)nonZero; }

	virtual int Solve(const LinearSolverSettings &ls, CRS_Matrix &crs, Vector<double> &rhs,
	                  Vector<double> &x, int &iter, double &resid)
	{
		const int n = crs.RowSize(), nnz = crs.NonZero();
		if(n != _n || nnz != _nnz || !SamePattern(crs))
		{
			if(yz_solver_set_pattern(_s, n, nnz, crs.RowPtrData(), crs.SortedColIndData(), crs.SortedSrcData()) != 0)
				throw std::runtime_error(std::string("b200 backend: ") + yz_last_error());
			_n = n; _nnz = nnz;
			_rowptr.assign(crs.RowPtrData(), crs.RowPtrData() + n + 1);
			_col.assign(crs.ColIndData(), crs.ColIndData() + nnz);
		}
		yz_settings s;
		s.precondition = (int)ls.precondition;
		s.scaling = ls.scaling ? 1 : 0;
		s.max_iteration = ls.maxIteration;
		s.epsilon = ls.epsilon;
		s.conc = ls.conc ? 1 : 0;
		const int ret = yz_solver_solve(_s, &s, crs.ValuesData(), rhs.data(), x.data(), &iter, &resid);
		if(ret < 0) throw std::runtime_error(std::string("b200 backend: ") + yz_last_error());
		return ret;
	}

	virtual std::vector<double> Memory() const
	{
		double m[8];
		const int k = yz_solver_memory(_s, m, 8);
		return std::vector<double>(m, m + (k > 0 ? k : 0));
	}
	virtual void SetMemory(const std::vector<double> &m) { yz_solver_set_memory(_s, m.data(), (int)m.size()); }

private:
	bool SamePattern(const CRS_Matrix &crs) const
	{
		const int *rp = crs.RowPtrData(), *c = crs.ColIndData();
		for(int i = 0; i <= _n; ++i) if(rp[i] != _rowptr[(size_t)i]) return false;
		for(int k = 0; k < _nnz; ++k) if(c[k] != _col[(size_t)k]) return false;
		return true;
	}
	yz_solver *_s;
	int _n, _nnz;
	std::vector<int> _rowptr, _col;
};

} // namespace

ILinearSolverBackend* MakeB200LinearSolverBackend() { return new B200Backend(); }
