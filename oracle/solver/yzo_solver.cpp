/*
 * yzo_solver.cpp -- the CPU oracle of the linear solve (TEST INFRASTRUCTURE,
 * the checker of the CUDA solver; see yzo_solver.h).
 *
 * Every floating-point operation below is specified exactly, because the CUDA
 * solver reproduces it bit for bit (compiled without FMA contraction, like
 * this file: -ffp-contract=off, the flag of the reference's CMakeLists.txt:33-46).
 *
 *  Reductions (dot, norm). The reference's Vector<T> fixes its summation order
 *  by blocks (MyMath/Vector.h:55-71); AMGCL's builtin backend does not.  The
 *  order used here is a fixed tree that a GPU evaluates without atomics:
 *  chunks of 4096 elements; inside a chunk, "thread" t in 0..255 sums elements
 *  t, t+256, ..., t+15*256 sequentially from 0.0; the 256 sums are folded
 *  pairwise (s[t] += s[t+off] for off = 128, 64, ..., 1); the chunk sums are
 *  then folded the same way (thread t sums chunks t, t+256, ... from 0.0).
 *
 *  SpMV / residual (CRS_Matrix::MatVec, CRS_Matrix.cpp:307-329): per row, from
 *  0.0, in the stored order; residual r_i = f_i - (that sum).
 *
 *  Smoothed aggregation (AMGCL coarsening::smoothed_aggregation defaults:
 *  eps_strong 0.08 halved per level, relax 1, omega = 2/3, constant null
 *  space):
 *    strong(i,j), j != i:  (eps^2 * d_i) * d_j < a_ij^2, d the diagonal.
 *    aggregation: a distance-2 maximal independent set of the symmetrised
 *      strong graph (Bell, Dalton, Olson 2012), priorities from a fixed hash
 *      of the row number; roots numbered in row order; a row joins the
 *      aggregate of its adjacent root, else the smallest aggregate among its
 *      neighbours that joined in that first pass.  Rows with no strong
 *      connection in either direction join none.  AMGCL aggregates greedily
 *      in row order instead; the MIS-2 form is the one a GPU can build, and
 *      it is used on both sides.
 *    P = (I - omega D_f^-1 A_f) P_tent, A_f the strong part of A with the weak
 *      entries lumped into the diagonal; row i of P accumulates, from 0.0 and
 *      in the stored order of row i, (1 - omega) for the diagonal and
 *      (-omega * (1 / d_f)) * a_ij for a strong entry, into the aggregate of
 *      column j; P's rows are then sorted by column.  R = P^T.
 *    Galerkin product C = X Y: C_ij = sum over the stored k of row i of X, in
 *      ascending k, of X_ik * Y_kj, from 0.0; the pattern is the structural
 *      product; rows sorted.  A_c = R (A P).
 *    SPAI0: m_i = (1 / sum_j a_ij^2) * (0.0 + a_ii).
 *    The coarsest level (<= coarse_enough rows) is inverted by Gauss-Jordan
 *      on [A | I] with partial pivoting (first row of largest |a|; a row whose
 *      multiplier is 0.0 is skipped) and applied as a dense product summed in
 *      column order from 0.0.
 *  V-cycle, one pre- and one post-sweep of SPAI0 from a zero guess:
 *    x = m .* f; t = f - A x; f_c = R t; x_c = V(f_c); x = x + P x_c (the
 *    product summed from 0.0, then added); t = f - A x; x = x + m .* t.
 *  BiCGStab (van der Vorst 1992), right preconditioned as AMGCL's
 *    solver::bicgstab: see BiCGStab() below for the exact update order.
 */
#include "yzo_solver.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

namespace {

//--------------------------------------------------------------------------
//  deterministic reduction
//--------------------------------------------------------------------------
const int kRT = 256, kRK = 1, kRChunk = kRT * kRK;

double Tree256(double *s)
{
	for(int off = kRT / 2; off >= 1; off >>= 1)
		for(int t = 0; t < off; ++t) s[t] = s[t] + s[t + off];
	return s[0];
}

template<class F> double DetSum(int n, F f)
{
	const int nb = (n + kRChunk - 1) / kRChunk;
	std::vector<double> part((size_t)(nb > 0 ? nb : 1), 0.0);
	double s[kRT];
	//  the chunks' sums are independent, each its own fixed tree
#pragma omp parallel for schedule(static) if(nb > 16)
	for(int b = 0; b < nb; ++b)
	{
		double s[kRT];
		for(int t = 0; t < kRT; ++t)
		{
			double a = 0.0;
			for(int k = 0; k < kRK; ++k)
			{
				const long long i = (long long)b * kRChunk + (long long)k * kRT + t;
				if(i < n) a = a + f((int)i);
			}
			s[t] = a;
		}
		part[(size_t)b] = Tree256(s);
	}
#pragma omp parallel for schedule(static) if(nb > 4096)
	for(int t = 0; t < kRT; ++t)
	{
		double a = 0.0;
		for(int j = t; j < nb; j += kRT) a = a + part[(size_t)j];
		s[t] = a;
	}
	return Tree256(s);
}

double Dot(int n, const double *x, const double *y)
{
	return DetSum(n, [&](int i) { return x[i] * y[i]; });
}

//--------------------------------------------------------------------------
//  CSR (column-sorted rows except where noted)
//--------------------------------------------------------------------------
struct Csr
{
	int n = 0, m = 0;			// rows, columns
	std::vector<int> ptr, col;
	std::vector<double> val;
	int nnz() const { return ptr.empty() ? 0 : ptr[(size_t)n]; }
};

void Spmv(const Csr &A, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
	for(int i = 0; i < A.n; ++i)
	{
		double s = 0.0;
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k) s = s + A.val[(size_t)k] * x[A.col[(size_t)k]];
		y[i] = s;
	}
}

//  the restriction R t: each row as four strided partial sums (entries q,
//  q+4, ... of the row into partial q, from 0.0) folded (p0 + p1) + (p2 + p3),
//  the order the device's four lanes per row take
void Restrict(const Csr &R, const double *t, double *y)
{
#pragma omp parallel for schedule(static)
	for(int i = 0; i < R.n; ++i)
	{
		double p[4] = {0.0, 0.0, 0.0, 0.0};
		const int st = R.ptr[(size_t)i], ed = R.ptr[(size_t)i + 1];
		for(int k = st; k < ed; ++k) p[(k - st) & 3] = p[(k - st) & 3] + R.val[(size_t)k] * t[R.col[(size_t)k]];
		y[i] = (p[0] + p[1]) + (p[2] + p[3]);
	}
}

void Residual(const Csr &A, const double *f, const double *x, double *r)
{
#pragma omp parallel for schedule(static)
	for(int i = 0; i < A.n; ++i)
	{
		double s = 0.0;
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k) s = s + A.val[(size_t)k] * x[A.col[(size_t)k]];
		r[i] = f[i] - s;
	}
}

double DiagOf(const Csr &A, int i)
{
	for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
		if(A.col[(size_t)k] == i) return A.val[(size_t)k];
	return 0.0;
}

void Spai0(const Csr &A, std::vector<double> &M)
{
	M.assign((size_t)A.n, 0.0);
#pragma omp parallel for schedule(static)
	for(int i = 0; i < A.n; ++i)
	{
		double num = 0.0, den = 0.0;
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
		{
			const double v = A.val[(size_t)k];
			den = den + v * v;
			if(A.col[(size_t)k] == i) num = num + v;
		}
		M[(size_t)i] = (1.0 / den) * num;
	}
}

//  structural product with the summation order of the file header
void Multiply(const Csr &X, const Csr &Y, Csr &C)
{
	C.n = X.n; C.m = Y.m;
	C.ptr.assign((size_t)C.n + 1, 0);
	C.col.clear(); C.val.clear();
	//  every row on its own (rows in parallel, each with its own marker and
	//  accumulator), then the rows laid end to end
	std::vector<std::vector<int>> rc((size_t)X.n);
	std::vector<std::vector<double>> rv((size_t)X.n);
#pragma omp parallel
	{
		std::vector<int> marker((size_t)Y.m, -1);
		std::vector<double> acc((size_t)Y.m, 0.0);
		std::vector<int> cols;
#pragma omp for schedule(static)
		for(int i = 0; i < X.n; ++i)
		{
			cols.clear();
			for(int kx = X.ptr[(size_t)i]; kx < X.ptr[(size_t)i + 1]; ++kx)
			{
				const int k = X.col[(size_t)kx];
				const double xv = X.val[(size_t)kx];
				for(int ky = Y.ptr[(size_t)k]; ky < Y.ptr[(size_t)k + 1]; ++ky)
				{
					const int j = Y.col[(size_t)ky];
					if(marker[(size_t)j] != i) { marker[(size_t)j] = i; acc[(size_t)j] = 0.0; cols.push_back(j); }
					acc[(size_t)j] = acc[(size_t)j] + xv * Y.val[(size_t)ky];
				}
			}
			std::sort(cols.begin(), cols.end());
			rc[(size_t)i] = cols;
			rv[(size_t)i].resize(cols.size());
			for(size_t q = 0; q < cols.size(); ++q) rv[(size_t)i][q] = acc[(size_t)cols[q]];
		}
	}
	for(int i = 0; i < X.n; ++i) C.ptr[(size_t)i + 1] = C.ptr[(size_t)i] + (int)rc[(size_t)i].size();
	C.col.resize((size_t)C.ptr[(size_t)X.n]);
	C.val.resize((size_t)C.ptr[(size_t)X.n]);
#pragma omp parallel for schedule(static)
	for(int i = 0; i < X.n; ++i)
	{
		std::copy(rc[(size_t)i].begin(), rc[(size_t)i].end(), C.col.begin() + C.ptr[(size_t)i]);
		std::copy(rv[(size_t)i].begin(), rv[(size_t)i].end(), C.val.begin() + C.ptr[(size_t)i]);
	}
}

void Transpose(const Csr &P, Csr &R)
{
	R.n = P.m; R.m = P.n;
	R.ptr.assign((size_t)R.n + 1, 0);
	for(int k = 0; k < P.nnz(); ++k) R.ptr[(size_t)P.col[(size_t)k] + 1]++;
	for(int i = 0; i < R.n; ++i) R.ptr[(size_t)i + 1] += R.ptr[(size_t)i];
	R.col.assign((size_t)P.nnz(), 0);
	R.val.assign((size_t)P.nnz(), 0.0);
	std::vector<int> fill(R.ptr.begin(), R.ptr.end() - 1);
	for(int i = 0; i < P.n; ++i)
		for(int k = P.ptr[(size_t)i]; k < P.ptr[(size_t)i + 1]; ++k)
		{
			const int c = P.col[(size_t)k];
			const int d = fill[(size_t)c]++;
			R.col[(size_t)d] = i;
			R.val[(size_t)d] = P.val[(size_t)k];
		}
}

//--------------------------------------------------------------------------
//  aggregation
//--------------------------------------------------------------------------
uint32_t Hash32(uint32_t x)
{
	//  a fixed integer mixer (the 32-bit finaliser of MurmurHash3)
	x ^= x >> 16; x *= 0x85ebca6bu;
	x ^= x >> 13; x *= 0xc2b2ae35u;
	x ^= x >> 16;
	return x;
}

enum { kOut = 0, kUndecided = 1, kIn = 2 };
const int kMisMaxRounds = 64;

uint64_t Pack(int state, int i)
{
	return ((uint64_t)state << 62) | ((uint64_t)(Hash32((uint32_t)i) & 0x3fffffffu) << 32) | (uint64_t)(uint32_t)i;
}

//  strong flags per stored entry (directed), the diagonal per row
void Strength(const Csr &A, double eps, std::vector<char> &strong, std::vector<double> &dia)
{
	dia.assign((size_t)A.n, 0.0);
#pragma omp parallel for schedule(static)
	for(int i = 0; i < A.n; ++i) dia[(size_t)i] = DiagOf(A, i);
	strong.assign((size_t)A.nnz(), 0);
	const double eps2 = eps * eps;
#pragma omp parallel for schedule(static)
	for(int i = 0; i < A.n; ++i)
	{
		const double e = eps2 * dia[(size_t)i];
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
		{
			const int c = A.col[(size_t)k];
			const double v = A.val[(size_t)k];
			strong[(size_t)k] = (c != i) && (e * dia[(size_t)c] < v * v);
		}
	}
}

//  aggregate of every row (-1: none), and the number of aggregates
int Aggregate(const Csr &A, const std::vector<char> &strong, std::vector<int> &agg)
{
	const int n = A.n;
	//  the symmetrised strong graph: out-neighbours (the strong entries of
	//  the row) and in-neighbours (the rows holding this one strongly)
	std::vector<int> iptr((size_t)n + 1, 0), icol;
	for(int i = 0; i < n; ++i)
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
			if(strong[(size_t)k]) iptr[(size_t)A.col[(size_t)k] + 1]++;
	for(int i = 0; i < n; ++i) iptr[(size_t)i + 1] += iptr[(size_t)i];
	icol.assign((size_t)iptr[(size_t)n], 0);
	{
		std::vector<int> fill(iptr.begin(), iptr.end() - 1);
		for(int i = 0; i < n; ++i)
			for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
				if(strong[(size_t)k]) icol[(size_t)fill[(size_t)A.col[(size_t)k]]++] = i;
	}
	auto forNbr = [&](int i, auto fn) {
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
			if(strong[(size_t)k]) fn(A.col[(size_t)k]);
		for(int k = iptr[(size_t)i]; k < iptr[(size_t)i + 1]; ++k) fn(icol[(size_t)k]);
	};

	std::vector<int> state((size_t)n, kUndecided);
	std::vector<char> isolated((size_t)n, 1);
	for(int i = 0; i < n; ++i) { bool any = false; forNbr(i, [&](int) { any = true; }); isolated[(size_t)i] = any ? 0 : 1; if(!any) state[(size_t)i] = kOut; }

	std::vector<uint64_t> T0((size_t)n), T1((size_t)n), T2((size_t)n);
	for(int round = 0; round < kMisMaxRounds; ++round)
	{
		bool undecided = false;
		for(int i = 0; i < n; ++i) if(state[(size_t)i] == kUndecided) { undecided = true; break; }
		if(!undecided) break;
#pragma omp parallel for schedule(static)
		for(int i = 0; i < n; ++i) T0[(size_t)i] = Pack(state[(size_t)i], i);
#pragma omp parallel for schedule(static)
		for(int i = 0; i < n; ++i) { uint64_t m = T0[(size_t)i]; forNbr(i, [&](int j) { m = std::max(m, T0[(size_t)j]); }); T1[(size_t)i] = m; }
#pragma omp parallel for schedule(static)
		for(int i = 0; i < n; ++i) { uint64_t m = T1[(size_t)i]; forNbr(i, [&](int j) { m = std::max(m, T1[(size_t)j]); }); T2[(size_t)i] = m; }
#pragma omp parallel for schedule(static)
		for(int i = 0; i < n; ++i)
		{
			if(state[(size_t)i] != kUndecided) continue;
			if((int)(uint32_t)(T2[(size_t)i] & 0xffffffffu) == i) state[(size_t)i] = kIn;
			else if((int)(T2[(size_t)i] >> 62) == kIn) state[(size_t)i] = kOut;
		}
	}

	agg.assign((size_t)n, -1);
	int nc = 0;
	for(int i = 0; i < n; ++i) if(state[(size_t)i] == kIn) agg[(size_t)i] = nc++;
	//  first pass: the adjacent root
	std::vector<int> first(agg);
#pragma omp parallel for schedule(static)
	for(int i = 0; i < n; ++i)
	{
		if(state[(size_t)i] == kIn || isolated[(size_t)i]) continue;
		int best = -1;
		forNbr(i, [&](int j) { if(state[(size_t)j] == kIn && (best < 0 || agg[(size_t)j] < best)) best = agg[(size_t)j]; });
		first[(size_t)i] = best;
	}
	//  second pass: a neighbour placed by the first
	std::vector<int> second(first);
#pragma omp parallel for schedule(static)
	for(int i = 0; i < n; ++i)
	{
		if(first[(size_t)i] >= 0 || isolated[(size_t)i]) continue;
		int best = -1;
		forNbr(i, [&](int j) { if(first[(size_t)j] >= 0 && (best < 0 || first[(size_t)j] < best)) best = first[(size_t)j]; });
		second[(size_t)i] = best;
	}
	agg.swap(second);
	return nc;
}

//  the smoothed prolongation
void SmoothedP(const Csr &A, const std::vector<char> &strong, const std::vector<int> &agg, int nc, Csr &P)
{
	const double omega = 2.0 / 3.0;
	P.n = A.n; P.m = nc;
	P.ptr.assign((size_t)A.n + 1, 0);
	P.col.clear(); P.val.clear();
	//  every row on its own (rows in parallel), then laid end to end
	std::vector<std::vector<int>> rc((size_t)A.n);
	std::vector<std::vector<double>> rv((size_t)A.n);
#pragma omp parallel
	{
	std::vector<int> lc; std::vector<double> lv;
	std::vector<int> order;
#pragma omp for schedule(static)
	for(int i = 0; i < A.n; ++i)
	{
		double dia = 0.0;
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
			if(A.col[(size_t)k] == i || !strong[(size_t)k]) dia = dia + A.val[(size_t)k];
		const double ds = (-omega) * (1.0 / dia);
		lc.clear(); lv.clear();
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k)
		{
			const int c = A.col[(size_t)k];
			if(c != i && !strong[(size_t)k]) continue;
			const int cp = agg[(size_t)c];
			if(cp < 0) continue;
			const double va = (c == i) ? (1.0 - omega) : ds * A.val[(size_t)k];
			size_t q = 0;
			while(q < lc.size() && lc[q] != cp) ++q;
			if(q == lc.size()) { lc.push_back(cp); lv.push_back(0.0); }
			lv[q] = lv[q] + va;
		}
		order.resize(lc.size());
		for(size_t q = 0; q < lc.size(); ++q) order[q] = (int)q;
		std::sort(order.begin(), order.end(), [&](int a, int b) { return lc[(size_t)a] < lc[(size_t)b]; });
		for(int q : order) { rc[(size_t)i].push_back(lc[(size_t)q]); rv[(size_t)i].push_back(lv[(size_t)q]); }
	}
	}
	for(int i = 0; i < A.n; ++i) P.ptr[(size_t)i + 1] = P.ptr[(size_t)i] + (int)rc[(size_t)i].size();
	P.col.resize((size_t)P.ptr[(size_t)A.n]);
	P.val.resize((size_t)P.ptr[(size_t)A.n]);
#pragma omp parallel for schedule(static)
	for(int i = 0; i < A.n; ++i)
	{
		std::copy(rc[(size_t)i].begin(), rc[(size_t)i].end(), P.col.begin() + P.ptr[(size_t)i]);
		std::copy(rv[(size_t)i].begin(), rv[(size_t)i].end(), P.val.begin() + P.ptr[(size_t)i]);
	}
}

void GaussJordanInverse(const Csr &A, std::vector<double> &inv)
{
	const int n = A.n, w = 2 * n;
	std::vector<double> M((size_t)n * w, 0.0);
	for(int i = 0; i < n; ++i)
	{
		for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k) M[(size_t)i * w + A.col[(size_t)k]] = A.val[(size_t)k];
		M[(size_t)i * w + n + i] = 1.0;
	}
	for(int k = 0; k < n; ++k)
	{
		int p = k;
		double best = std::fabs(M[(size_t)k * w + k]);
		for(int i = k + 1; i < n; ++i)
		{
			const double a = std::fabs(M[(size_t)i * w + k]);
			if(a > best) { best = a; p = i; }
		}
		if(p != k)
			for(int j = 0; j < w; ++j) std::swap(M[(size_t)k * w + j], M[(size_t)p * w + j]);
		const double piv = M[(size_t)k * w + k];
		for(int j = 0; j < w; ++j) M[(size_t)k * w + j] = M[(size_t)k * w + j] / piv;
#pragma omp parallel for schedule(static) if(n > 64)
		for(int i = 0; i < n; ++i)
		{
			if(i == k) continue;
			const double f = M[(size_t)i * w + k];
			if(f == 0.0) continue;
			for(int j = 0; j < w; ++j) M[(size_t)i * w + j] = M[(size_t)i * w + j] - f * M[(size_t)k * w + j];
		}
	}
	inv.assign((size_t)n * n, 0.0);
	for(int i = 0; i < n; ++i)
		for(int j = 0; j < n; ++j) inv[(size_t)i * n + j] = M[(size_t)i * w + n + j];
}

//--------------------------------------------------------------------------
//  the hierarchy and the V-cycle
//--------------------------------------------------------------------------
struct Level
{
	Csr A, P, R;
	std::vector<double> M;			// SPAI0
	std::vector<int> agg;
	bool direct = false;
	std::vector<double> inv;		// dense inverse of the direct level
	std::vector<double> f, x, t;	// work
};

struct Hierarchy
{
	std::vector<Level> lv;

	void Build(const Csr &A0, int coarseEnough)
	{
		lv.clear();
		lv.emplace_back();
		lv.back().A = A0;
		double eps = 0.08;
		for(;;)
		{
			Level &L = lv.back();
			if(L.A.n <= coarseEnough)
			{
				L.direct = true;
				GaussJordanInverse(L.A, L.inv);
				break;
			}
			std::vector<char> strong; std::vector<double> dia;
			Strength(L.A, eps, strong, dia);
			eps *= 0.5;
			const int nc = Aggregate(L.A, strong, L.agg);
			Spai0(L.A, L.M);
			if(nc == 0) break;				// nothing to coarsen: smoothed only
			SmoothedP(L.A, strong, L.agg, nc, L.P);
			Transpose(L.P, L.R);
			Csr AP, Ac;
			Multiply(L.A, L.P, AP);
			Multiply(L.R, AP, Ac);
			lv.emplace_back();
			lv.back().A = std::move(Ac);
		}
		for(Level &L : lv)
		{
			L.f.assign((size_t)L.A.n, 0.0); L.x.assign((size_t)L.A.n, 0.0); L.t.assign((size_t)L.A.n, 0.0);
		}
	}

	//  x = V(l) f, from a zero guess
	void Cycle(size_t l, const double *f, double *x)
	{
		Level &L = lv[l];
		const int n = L.A.n;
		if(L.direct)
		{
			//  row i of the inverse times f as 32 strided partial sums
			//  (lane l: j = l, l+32, ... from 0.0) folded pairwise
#pragma omp parallel for schedule(static) if(n > 64)
			for(int i = 0; i < n; ++i)
			{
				double s[32];
				const double *row = &L.inv[(size_t)i * n];
				for(int l = 0; l < 32; ++l)
				{
					double a = 0.0;
					for(int j = l; j < n; j += 32) a = a + row[j] * f[j];
					s[l] = a;
				}
				for(int off = 16; off >= 1; off >>= 1)
					for(int l = 0; l < off; ++l) s[l] = s[l] + s[l + off];
				x[i] = s[0];
			}
			return;
		}
#pragma omp parallel for schedule(static)
		for(int i = 0; i < n; ++i) x[i] = L.M[(size_t)i] * f[i];
		Residual(L.A, f, x, L.t.data());
		if(l + 1 < lv.size())
		{
			Level &C = lv[l + 1];
			Restrict(L.R, L.t.data(), C.f.data());
			Cycle(l + 1, C.f.data(), C.x.data());
#pragma omp parallel for schedule(static)
			for(int i = 0; i < n; ++i)
			{
				double s = 0.0;
				for(int k = L.P.ptr[(size_t)i]; k < L.P.ptr[(size_t)i + 1]; ++k) s = s + L.P.val[(size_t)k] * C.x[(size_t)L.P.col[(size_t)k]];
				x[i] = x[i] + s;
			}
			Residual(L.A, f, x, L.t.data());
		}
#pragma omp parallel for schedule(static)
		for(int i = 0; i < n; ++i) x[i] = x[i] + L.M[(size_t)i] * L.t[(size_t)i];
	}
};

//--------------------------------------------------------------------------
//  ILU(0) on the sorted pattern (the Eigen flavour only)
//--------------------------------------------------------------------------
struct Ilu0
{
	Csr LU;
	std::vector<int> dpos;
	bool Setup(const Csr &A)
	{
		LU = A;
		const int n = A.n;
		dpos.assign((size_t)n, -1);
		for(int i = 0; i < n; ++i)
			for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k) if(A.col[(size_t)k] == i) dpos[(size_t)i] = k;
		for(int i = 0; i < n; ++i) if(dpos[(size_t)i] < 0) return false;
		for(int i = 1; i < n; ++i)
		{
			for(int k = LU.ptr[(size_t)i]; k < LU.ptr[(size_t)i + 1]; ++k)
			{
				const int kk = LU.col[(size_t)k];
				if(kk >= i) break;
				const double dkk = LU.val[(size_t)dpos[(size_t)kk]];
				if(dkk == 0.0) return false;
				LU.val[(size_t)k] = LU.val[(size_t)k] / dkk;
				const double lik = LU.val[(size_t)k];
				for(int j = k + 1; j < LU.ptr[(size_t)i + 1]; ++j)
				{
					const int cj = LU.col[(size_t)j];
					for(int q = dpos[(size_t)kk] + 1; q < LU.ptr[(size_t)kk + 1]; ++q)
						if(LU.col[(size_t)q] == cj) { LU.val[(size_t)j] = LU.val[(size_t)j] - lik * LU.val[(size_t)q]; break; }
				}
			}
		}
		for(int i = 0; i < n; ++i) if(LU.val[(size_t)dpos[(size_t)i]] == 0.0) return false;
		return true;
	}
	void Apply(const double *r, double *z) const
	{
		const int n = LU.n;
		for(int i = 0; i < n; ++i)
		{
			double s = r[i];
			for(int k = LU.ptr[(size_t)i]; k < dpos[(size_t)i]; ++k) s = s - LU.val[(size_t)k] * z[LU.col[(size_t)k]];
			z[i] = s;
		}
		for(int i = n - 1; i >= 0; --i)
		{
			double s = z[i];
			for(int k = dpos[(size_t)i] + 1; k < LU.ptr[(size_t)i + 1]; ++k) s = s - LU.val[(size_t)k] * z[LU.col[(size_t)k]];
			z[i] = s / LU.val[(size_t)dpos[(size_t)i]];
		}
	}
};

//--------------------------------------------------------------------------
//  BiCGStab
//--------------------------------------------------------------------------
struct Breakdown : std::runtime_error { Breakdown() : std::runtime_error("Zero rho in BiCGStab") {} };

template<class Prec>
void BiCGStab(const Csr &A, Prec &&prec, const double *b, double *x, int maxIter, double tol,
              int &itOut, double &errOut)
{
	const int n = A.n;
	std::vector<double> r((size_t)n), rh((size_t)n), p((size_t)n), v((size_t)n), s((size_t)n),
	                    ph((size_t)n), sh((size_t)n), t((size_t)n);
	Residual(A, b, x, r.data());
	const double normB = std::sqrt(Dot(n, b, b));
	if(normB < 2.0 * 2.220446049250313e-16)
	{
		for(int i = 0; i < n; ++i) x[i] = 0.0;
		itOut = 0; errOut = normB;
		return;
	}
	const double eps = tol * normB;
	double res = std::sqrt(Dot(n, r.data(), r.data()));
	int it = 0;
	if(res > eps)
	{
		rh = r;
		double rhoPrev = 1.0, alpha = 1.0, omega = 1.0;
		while(it < maxIter)
		{
			const double rho = Dot(n, rh.data(), r.data());
			if(rho == 0.0) throw Breakdown();
			if(it == 0) p = r;
			else
			{
				const double beta = (rho / rhoPrev) * (alpha / omega);
#pragma omp parallel for schedule(static)
				for(int i = 0; i < n; ++i) p[(size_t)i] = r[(size_t)i] + beta * (p[(size_t)i] - omega * v[(size_t)i]);
			}
			prec(p.data(), ph.data());
			Spmv(A, ph.data(), v.data());
			alpha = rho / Dot(n, rh.data(), v.data());
#pragma omp parallel for schedule(static)
			for(int i = 0; i < n; ++i) s[(size_t)i] = r[(size_t)i] - alpha * v[(size_t)i];
			res = std::sqrt(Dot(n, s.data(), s.data()));
			if(res <= eps)
			{
				for(int i = 0; i < n; ++i) x[i] = x[i] + alpha * ph[(size_t)i];
				++it;
				break;
			}
			prec(s.data(), sh.data());
			Spmv(A, sh.data(), t.data());
			const double tt = Dot(n, t.data(), t.data());
			const double ts = Dot(n, t.data(), s.data());
			omega = ts / tt;
#pragma omp parallel for schedule(static)
			for(int i = 0; i < n; ++i) x[i] = (x[i] + alpha * ph[(size_t)i]) + omega * sh[(size_t)i];
#pragma omp parallel for schedule(static)
			for(int i = 0; i < n; ++i) r[(size_t)i] = s[(size_t)i] - omega * t[(size_t)i];
			rhoPrev = rho;
			res = std::sqrt(Dot(n, r.data(), r.data()));
			++it;
			if(res <= eps) break;
			if(!(res == res)) break;
		}
	}
	itOut = it;
	errOut = res / normB;
}

//  TryBackoff, LinearSolverBackend.cpp:262-270
struct TryBackoff
{
	int skip = 0, wait = 16;
	bool Try() { if(skip > 0) { --skip; return false; } return true; }
	void Failed() { skip = wait; wait = (wait < 1024) ? 2 * wait : 1024; }
	void Converged() { wait = 16; }
};

} // namespace

//--------------------------------------------------------------------------
//  Fault injection (LinearSolverBackend.cpp:630-645): YUZEN_FAULT_AMGCL=k:m
//  makes m solves of the process, from the k-th on, that reach the AMG /
//  Jacobi path break down before they iterate (m = 1 if left out).  The
//  count is of the process, over every solver.
//--------------------------------------------------------------------------
struct Fault
{
	long at = 0, count = 0, solves = 0;
	Fault()
	{
		if(const char *e = std::getenv("YUZEN_FAULT_AMGCL"))
		{
			char *end = nullptr;
			at = std::strtol(e, &end, 10);
			count = (end && *end == ':') ? std::strtol(end + 1, nullptr, 10) : 1;
		}
	}
	bool Now() { return at > 0 && ++solves >= at && solves < at + count; }
};
Fault &TheFault() { static Fault f; return f; }

//==========================================================================
struct yzo_solver
{
	int flavour;
	TryBackoff offFirst, offBlock;		// SPAI0 / Jacobi try (concpc); block ILUT (unused)
	Hierarchy H;
	bool haveH = false;
	std::vector<double> val, b, xx;
};

extern "C" {

yzo_solver* yzo_create(int flavour)
{
	yzo_solver *s = new yzo_solver();
	s->flavour = flavour;
	return s;
}

void yzo_destroy(yzo_solver *s) { delete s; }

double yzo_dot(int n, const double *x, const double *y) { return Dot(n, x, y); }

void yzo_spmv(int n, const int *rowptr, const int *col, const double *val, const double *x, double *y)
{
	for(int i = 0; i < n; ++i)
	{
		double s = 0.0;
		for(int k = rowptr[i]; k < rowptr[i + 1]; ++k) s = s + val[k] * x[col[k]];
		y[i] = s;
	}
}

int yzo_solve(yzo_solver *S, const yzo_settings *set, int n,
              const int *rowptr, const int *scol, const int *ssrc,
              const double *values, const double *rhs, double *x,
              int *iterOut, double *residOut)
{
	const int nnz = rowptr[n];
	Csr A;
	A.n = n; A.m = n;
	A.ptr.assign(rowptr, rowptr + n + 1);
	A.col.assign(scol, scol + nnz);
	A.val.assign((size_t)nnz, 0.0);
	S->b.assign((size_t)n, 0.0);
	S->xx.assign(x, x + n);
	//  ScaleRows, LinearSolverBackend.cpp:227-252
#pragma omp parallel for schedule(static)
	for(int i = 0; i < n; ++i)
	{
		const int st = rowptr[i], ed = rowptr[i + 1];
		const double d = set->scaling ? values[st] : 1.0;
		if(!set->scaling || std::fabs(d) < 1.0e-30)
		{
			for(int k = st; k < ed; ++k) A.val[(size_t)k] = values[ssrc[k]];
			S->b[(size_t)i] = rhs[i];
			continue;
		}
		const double inv = 1.0 / d;
		for(int k = st; k < ed; ++k) A.val[(size_t)k] = values[ssrc[k]] * inv;
		S->b[(size_t)i] = rhs[i] * inv;
	}
	double *xx = S->xx.data();
	const double *b = S->b.data();
	int it = 0, itTried = 0;
	double err = 0.0;
	const int tryIter = set->max_iteration < 300 ? set->max_iteration : 300;

	if(S->flavour == YZO_ILU0)
	{
		//  EigenBackend::Solve, LinearSolverBackend.cpp:370-463 (ILU(0) for ILUT)
		auto runJacobi = [&](int maxIt) {
			std::vector<double> m((size_t)n);
			for(int i = 0; i < n; ++i) { const double d = DiagOf(A, i); m[(size_t)i] = (d == 0.0) ? 1.0 : 1.0 / d; }
			BiCGStab(A, [&](const double *r, double *z) { for(int i = 0; i < n; ++i) z[i] = m[(size_t)i] * r[i]; },
			         b, xx, maxIt, set->epsilon, it, err);
		};
		auto code = [&]() { if(err <= set->epsilon) return 0; if(!(err == err)) return 2; return 1; };
		try
		{
			if(set->conc && set->precondition == YZO_PC_ILU && S->offFirst.Try())
			{
				runJacobi(tryIter);
				if(code() == 0) { S->offFirst.Converged(); for(int i = 0; i < n; ++i) x[i] = xx[i]; *iterOut = it; *residOut = err; return 0; }
				S->offFirst.Failed();
				itTried += it;
				for(int i = 0; i < n; ++i) xx[i] = x[i];
			}
			if(set->precondition == YZO_PC_NONE)
				BiCGStab(A, [&](const double *r, double *z) { for(int i = 0; i < n; ++i) z[i] = r[i]; },
				         b, xx, set->max_iteration, set->epsilon, it, err);
			else if(set->precondition == YZO_PC_JACOBI) runJacobi(set->max_iteration);
			else
			{
				Ilu0 ilu;
				if(!ilu.Setup(A)) { *iterOut = itTried; *residOut = 0; return 2; }
				BiCGStab(A, [&](const double *r, double *z) { ilu.Apply(r, z); }, b, xx, set->max_iteration, set->epsilon, it, err);
			}
		}
		catch(const Breakdown &) { *iterOut = it + itTried; *residOut = err; return 2; }
		for(int i = 0; i < n; ++i) x[i] = xx[i];
		*iterOut = it + itTried;
		*residOut = err;
		return code();
	}

	//  AmgclBackend::Solve, LinearSolverBackend.cpp:539-728
	bool done = false;
	if(set->conc && set->precondition == YZO_PC_ILU && S->offFirst.Try())
	{
		std::vector<double> m;
		Spai0(A, m);
		try
		{
			BiCGStab(A, [&](const double *r, double *z) { for(int i = 0; i < n; ++i) z[i] = m[(size_t)i] * r[i]; },
			         b, xx, tryIter, set->epsilon, it, err);
		}
		catch(const Breakdown &) { err = 1e300; }
		if(err <= set->epsilon) { done = true; S->offFirst.Converged(); }
		else
		{
			S->offFirst.Failed();
			itTried = it;
			for(int i = 0; i < n; ++i) xx[i] = x[i];
		}
	}
	bool broke = false;
	if(!done && TheFault().Now()) broke = true;
	else if(!done)
	{
		try
		{
			if(set->precondition == YZO_PC_NONE || set->precondition == YZO_PC_JACOBI)
			{
				std::vector<double> m((size_t)n);
				for(int i = 0; i < n; ++i) m[(size_t)i] = 0.72 * (1.0 / DiagOf(A, i));
				BiCGStab(A, [&](const double *r, double *z) { for(int i = 0; i < n; ++i) z[i] = m[(size_t)i] * r[i]; },
				         b, xx, set->max_iteration, set->epsilon, it, err);
			}
			else
			{
				const int coarseEnough = (n > 3000) ? 500 : 3000;
				S->H.Build(A, coarseEnough);
				S->haveH = true;
				BiCGStab(A, [&](const double *r, double *z) { S->H.Cycle(0, r, z); },
				         b, xx, set->max_iteration, set->epsilon, it, err);
			}
		}
		catch(const Breakdown &) { broke = true; }
	}
	if(broke)
	{
		//  LinearSolverBackend.cpp:681-713: the residual of what x holds
		double rr = 0.0, bb = 0.0;
		for(int i = 0; i < n; ++i)
		{
			double ax = 0.0;
			for(int k = A.ptr[(size_t)i]; k < A.ptr[(size_t)i + 1]; ++k) ax += A.val[(size_t)k] * xx[A.col[(size_t)k]];
			const double d = b[i] - ax;
			rr += d * d; bb += b[i] * b[i];
		}
		const double rel = (bb > 0.0) ? std::sqrt(rr / bb) : std::sqrt(rr);
		if(rel <= set->epsilon && rel == rel) { it = 0; err = rel; }
		else { *iterOut = itTried; *residOut = rel; return 2; }
	}
	for(int i = 0; i < n; ++i) x[i] = xx[i];
	*iterOut = it + itTried;
	*residOut = err;
	if(err <= set->epsilon) return 0;
	if(!(err == err)) return 2;
	return 1;
}

void yzo_fault_inject(long at, long count)
{
	Fault &f = TheFault();
	f.at = at; f.count = count; f.solves = 0;
}

int yzo_memory(const yzo_solver *s, double *out, int cap)
{
	std::vector<double> m;
	m.push_back(s->offFirst.skip); m.push_back(s->offFirst.wait);
	if(s->flavour == YZO_ILU0) { m.push_back(s->offBlock.skip); m.push_back(s->offBlock.wait); }
	for(int i = 0; i < (int)m.size() && i < cap; ++i) out[i] = m[(size_t)i];
	return (int)m.size();
}

void yzo_set_memory(yzo_solver *s, const double *m, int len)
{
	const int want = (s->flavour == YZO_ILU0) ? 4 : 2;
	if(len != want) return;
	s->offFirst.skip = (int)m[0]; s->offFirst.wait = (int)m[1];
	if(want == 4) { s->offBlock.skip = (int)m[2]; s->offBlock.wait = (int)m[3]; }
}

int yzo_levels(const yzo_solver *s) { return s->haveH ? (int)s->H.lv.size() : 0; }

int yzo_level_info(const yzo_solver *s, int l, int *rows, int *nnzA, int *nnzP, int *direct)
{
	if(!s->haveH || l < 0 || l >= (int)s->H.lv.size()) return -1;
	const Level &L = s->H.lv[(size_t)l];
	if(rows) *rows = L.A.n;
	if(nnzA) *nnzA = L.A.nnz();
	if(nnzP) *nnzP = L.P.ptr.empty() ? 0 : L.P.nnz();
	if(direct) *direct = L.direct ? 1 : 0;
	return 0;
}

int yzo_level_copy(const yzo_solver *s, int l, int *aptr, int *acol, double *aval,
                   int *pptr, int *pcol, double *pval, int *agg)
{
	if(!s->haveH || l < 0 || l >= (int)s->H.lv.size()) return -1;
	const Level &L = s->H.lv[(size_t)l];
	if(aptr) std::copy(L.A.ptr.begin(), L.A.ptr.end(), aptr);
	if(acol) std::copy(L.A.col.begin(), L.A.col.end(), acol);
	if(aval) std::copy(L.A.val.begin(), L.A.val.end(), aval);
	if(!L.P.ptr.empty())
	{
		if(pptr) std::copy(L.P.ptr.begin(), L.P.ptr.end(), pptr);
		if(pcol) std::copy(L.P.col.begin(), L.P.col.end(), pcol);
		if(pval) std::copy(L.P.val.begin(), L.P.val.end(), pval);
	}
	if(agg && !L.agg.empty()) std::copy(L.agg.begin(), L.agg.end(), agg);
	return 0;
}

} // extern "C"
