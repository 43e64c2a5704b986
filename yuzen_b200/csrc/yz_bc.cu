// yz_bc.cu -- the host side of yz_bc.h: the ghost rows of BoundaryCondition2D
// written into a small row store that keeps the reference's storage order,
// and the SatisfyBCRows programme made from them.
#include "yz_bc.h"
#include "yz_common.cuh"

#include <algorithm>
#include <cmath>
#include <string>

namespace yz {
namespace {


//  a CRS row as the reference's CRS_Matrix keeps it: a diagonal slot first,
//  then the other columns in the order they were first written
struct Row
{
	bool any = false;
	double diag = 0.0;
	std::vector<int> col;
	std::vector<double> val;
	double rhs = 0.0;
};

struct Rows
{
	std::vector<Row> r;
	explicit Rows(int n) : r((size_t)n) {}
	void Diag(int i, double v) { r[(size_t)i].any = true; r[(size_t)i].diag = v; }
	void Set(int i, int j, double v)
	{
		if(j == i) { Diag(i, v); return; }
		Row &w = r[(size_t)i];
		w.any = true;
		for(size_t k = 0; k < w.col.size(); ++k)
			if(w.col[k] == j) { w.val[k] = v; return; }
		w.col.push_back(j);
		w.val.push_back(v);
	}
	void Rhs(int i, double v) { r[(size_t)i].rhs = v; }
};

//  the four-point rows of BoundaryCondition.cpp:22-79: columns cs, cs + st,
//  cs + 2 st, cs + 3 st
void FourPoint(Rows &w, int i, int cs, int st, const double c[4], double rhs)
{
	for(int k = 0; k < 4; ++k) w.Set(i, cs + k * st, c[k]);
	w.Rhs(i, rhs);
}
void Dirichlet(Rows &w, int i, int cs, int st, double b)
{
	const double c[4] = {-1.0 / 16.0, +9.0 / 16.0, +9.0 / 16.0, -1.0 / 16.0};
	FourPoint(w, i, cs, st, c, b);
}
void Derive2(Rows &w, int i, int cs, int st)
{
	const double c[4] = {+1.0 / 2.0, -1.0 / 2.0, -1.0 / 2.0, +1.0 / 2.0};
	const double dx = 0.0, b = 0.0;
	FourPoint(w, i, cs, st, c, dx * dx * b);
}
void Derive3(Rows &w, int i, int cs, int st)
{
	const double c[4] = {-1.0, +3.0, -3.0, +1.0};
	const double dx = 0.0, b = 0.0;
	FourPoint(w, i, cs, st, c, dx * dx * dx * b);
}
void EqualVal(Rows &w, int i, int j)
{
	w.Diag(i, 1.0);
	w.Set(i, j, -1.0);
	w.Rhs(i, 0.0);
}

//  one edge's two ghost rows (ApplyEdge): L[0] the outer ghost, L[3] the
//  second interior cell; opp the opposite edge's; cs, st the four-point
//  rows' first column and stride
struct Slot
{
	int L[4], opp[4], cs, st;
	double cb;      // the concentration the FreshInlet holds (the start field's, next to the edge)
};

void ApplyEdge(Rows &w, int tf, int tbc, const Slot &e)
{
	const int *L = e.L;
	switch(tbc)
	{
	default:
	case kBcSymmetry:
		EqualVal(w, L[0], L[3]);
		EqualVal(w, L[1], L[2]);
		break;
	case kBcPeriodic:
		EqualVal(w, L[0], e.opp[3]);
		EqualVal(w, L[1], e.opp[2]);
		break;
	case kBcPinning:
		if(tf == kBcFieldConc)
		{
			//  the concentration copied outwards (the 2-D form)
			EqualVal(w, L[1], L[2]);
			EqualVal(w, L[0], L[1]);
			break;
		}
		//  the film on the wall face zero, no normal velocity
		w.Diag(L[1], 0.5); w.Set(L[1], L[2], 0.5);
		w.Diag(L[0], 1.0); w.Set(L[0], L[1], -3.0); w.Set(L[0], L[2], +3.0); w.Set(L[0], L[3], -1.0);
		break;
	case kBcFreshInlet:
		if(tf == kBcFieldConc)
		{
			//  the start concentration at the edge held, zero second difference
			Dirichlet(w, L[1], e.cs, e.st, e.cb);
			w.Diag(L[0], 1.0); w.Set(L[0], L[1], -2.0); w.Set(L[0], L[2], +1.0);
			break;
		}
		//  the film's start value held (its right-hand side does not enter
		//  the pattern; the correction's is zero)
		Dirichlet(w, L[1], e.cs, e.st, 0.0);
		Derive3(w, L[0], e.cs, e.st);
		break;
	case kBcOutlet:
		Derive2(w, L[0], e.cs, e.st);
		Derive3(w, L[1], e.cs, e.st);
		break;
	}
}

//  the sixteen cells of a corner (BoundaryCondition.h stCornerIndex): the
//  upper-case pair says outside (O, a ghost layer) or inside (I) in x then
//  y, the lower-case pair the outer or inner of the two
struct Corner
{
	int OIoi, OIii, IIoi, IIii, OIoo, OIio, IIoo, IIio, OOoi, OOii, IOoi, IOii, OOoo, OOio, IOoo, IOio;
};

//  x0..x3 and y0..y3 run from the corner's outermost cell inwards
Corner MakeCorner(int nx, const int x[4], const int y[4])
{
	auto il = [nx](int ix, int iy) { return iy * nx + ix; };
	Corner c;
	c.OIoi = il(x[0], y[3]); c.OIii = il(x[1], y[3]); c.IIoi = il(x[2], y[3]); c.IIii = il(x[3], y[3]);
	c.OIoo = il(x[0], y[2]); c.OIio = il(x[1], y[2]); c.IIoo = il(x[2], y[2]); c.IIio = il(x[3], y[2]);
	c.OOoi = il(x[0], y[1]); c.OOii = il(x[1], y[1]); c.IOoi = il(x[2], y[1]); c.IOii = il(x[3], y[1]);
	c.OOoo = il(x[0], y[0]); c.OOio = il(x[1], y[0]); c.IOoo = il(x[2], y[0]); c.IOio = il(x[3], y[0]);
	return c;
}

void CopyCorner(Rows &w, const Corner &ci, int sii, int sio, int soi, int soo)
{
	EqualVal(w, ci.OOii, sii);
	EqualVal(w, ci.OOio, sio);
	EqualVal(w, ci.OOoi, soi);
	EqualVal(w, ci.OOoo, soo);
}
void MirrorXY(Rows &w, const Corner &ci, const Corner &cs) { CopyCorner(w, ci, cs.IIoo, cs.IIoi, cs.IIio, cs.IIii); }
void MirrorX(Rows &w, const Corner &ci, const Corner &cs) { CopyCorner(w, ci, cs.IOoi, cs.IOoo, cs.IOii, cs.IOio); }
void MirrorY(Rows &w, const Corner &ci, const Corner &cs) { CopyCorner(w, ci, cs.OIio, cs.OIii, cs.OIoo, cs.OIoi); }

//  the five-point corner rows, in the order OOoo, OOio, OOoi, OOii:
//  diagonal, then IIii, IIio, IIoi, IIoo, and the right-hand side's factor
//  of the corner value (BoundaryCondition.cpp:556-597)
struct CornerRow
{
	double d, cII, cIo, coI, coo, r;
};
const CornerRow kInletInletH[4] = {{-1.0, +4.0, -18.0, -18.0, +81.0, -(16.0 - 72.0 + 8.0)},
                                   {-3.0, +2.0, -9.0, -12.0, +54.0, -(8.0 - 48.0 + 8.0)},
                                   {-3.0, +2.0, -12.0, -9.0, +54.0, -(16.0 - 72.0 + 24.0)},
                                   {-9.0, +1.0, -6.0, -6.0, +36.0, -(8.0 - 48.0 + 24.0)}};
const CornerRow kInletInletC[4] = {{-49.0, +4.0, -54.0, -54.0, +729.0, -(64.0 - 864.0 + 224.0)},
                                   {-49.0, +2.0, -27.0, -20.0, +270.0, -(32.0 - 320.0 + 112.0)},
                                   {-49.0, +2.0, -20.0, -27.0, +270.0, -(32.0 - 432.0 + 224.0)},
                                   {-49.0, +1.0, -10.0, -10.0, +100.0, -(16.0 - 160.0 + 112.0)}};
const CornerRow kInletOutlet[4] = {{-1.0, -4.0, +6.0, +18.0, -27.0, -8.0},
                                   {-3.0, -2.0, +3.0, +12.0, -18.0, -8.0},
                                   {-1.0, -2.0, +4.0, +9.0, -18.0, -8.0},
                                   {-3.0, -1.0, +2.0, +6.0, -12.0, -8.0}};
const CornerRow kOutletInlet[4] = {{-1.0, -4.0, +18.0, +6.0, -27.0, -(-16.0 + 24.0)},
                                   {-1.0, -2.0, +9.0, +4.0, -18.0, -(-8.0 + 16.0)},
                                   {-3.0, -2.0, +12.0, +3.0, -18.0, -(-16.0 + 24.0)},
                                   {-3.0, -1.0, +6.0, +2.0, -12.0, -(-8.0 + 16.0)}};
const CornerRow kOutletOutlet[4] = {{-1.0, +4.0, -6.0, -6.0, +9.0, 0.0},
                                    {-1.0, +2.0, -3.0, -4.0, +6.0, 0.0},
                                    {-1.0, +2.0, -4.0, -3.0, +6.0, 0.0},
                                    {-1.0, +1.0, -2.0, -2.0, +4.0, 0.0}};

void CornerStencil(Rows &w, const Corner &ci, const CornerRow row[4], double val, bool setRhs)
{
	const int r[4] = {ci.OOoo, ci.OOio, ci.OOoi, ci.OOii};
	for(int k = 0; k < 4; ++k)
	{
		w.Diag(r[k], row[k].d);
		w.Set(r[k], ci.IIii, row[k].cII);
		w.Set(r[k], ci.IIio, row[k].cIo);
		w.Set(r[k], ci.IIoi, row[k].coI);
		w.Set(r[k], ci.IIoo, row[k].coo);
		if(setRhs) w.Rhs(r[k], row[k].r * val);
	}
}

const char *BcName(int t)
{
	switch(t)
	{
	case kBcSymmetry: return "Symmetry";
	case kBcPeriodic: return "Periodic";
	case kBcPinning: return "Pinning";
	case kBcFreshInlet: return "FreshInlet";
	default: return "Outlet";
	}
}

//  ApplyCorners (BoundaryCondition.cpp:612-743) with the corner value val
//  (the correction's zero for the film; the start concentration's mean near
//  the corner for the concentration); the combinations the reference does
//  not implement are refused as it refuses them
void ApplyCorner(Rows &w, int tf, int tx, int ty, const Corner &ci, const Corner &ciRO, const Corner &ciOR,
                 const Corner &ciRR, double val)
{
	const bool conc = (tf == kBcFieldConc);
	auto refuse = [&]() {
		throw UsageError(std::string("step: a corner of a ") + BcName(tx) + " and a " + BcName(ty) +
		                 " edge is not implemented (BC: " + BcName(tx) + "-" + BcName(ty) + ")");
	};
	switch(tx)
	{
	default:
	case kBcSymmetry:
		if(ty == kBcSymmetry) MirrorXY(w, ci, ci);
		else if(ty == kBcPeriodic) MirrorXY(w, ci, ciOR);
		else MirrorX(w, ci, ci);
		break;
	case kBcPeriodic:
		if(ty == kBcSymmetry) MirrorXY(w, ci, ciRO);
		else if(ty == kBcPeriodic) MirrorXY(w, ci, ciRR);
		else MirrorX(w, ci, ciRO);
		break;
	case kBcPinning:
		if(ty == kBcSymmetry && conc) MirrorXY(w, ci, ci);
		else if(ty == kBcSymmetry)
		{
			w.Diag(ci.OOii, 0.5); w.Set(ci.OOii, ci.IIoo, 0.5);
			w.Diag(ci.OOio, 0.5); w.Set(ci.OOio, ci.IIoi, 0.5);
			w.Diag(ci.OOoi, 1.0); w.Set(ci.OOoi, ci.OIoo, -1.0);
			w.Diag(ci.OOoo, 1.0); w.Set(ci.OOoo, ci.OIoi, -1.0);
		}
		else if(ty == kBcPeriodic) MirrorY(w, ci, ciOR);
		else if(ty == kBcPinning && conc) CopyCorner(w, ci, ci.IIoo, ci.OOii, ci.OOii, ci.OOii);
		else if(ty == kBcPinning)
			throw UsageError("step: two Pinning edges meeting at a corner leave three of the corner's ghost "
			                 "rows without a condition in the reference (BoundaryCondition.cpp:678-689)");
		else refuse();
		break;
	case kBcFreshInlet:
		if(ty == kBcSymmetry) MirrorY(w, ci, ci);
		else if(ty == kBcPeriodic) MirrorY(w, ci, ciOR);
		else if(ty == kBcFreshInlet) CornerStencil(w, ci, conc ? kInletInletC : kInletInletH, val, true);
		else if(ty == kBcOutlet) CornerStencil(w, ci, kInletOutlet, val, true);
		else refuse();
		break;
	case kBcOutlet:
		if(ty == kBcSymmetry) MirrorY(w, ci, ci);
		else if(ty == kBcPeriodic) MirrorY(w, ci, ciOR);
		else if(ty == kBcFreshInlet) CornerStencil(w, ci, kOutletInlet, val, true);
		else if(ty == kBcOutlet) CornerStencil(w, ci, kOutletOutlet, val, false);
		else refuse();
		break;
	}
}

void ApplyAll(Rows &w, const yz_step_params &p, int tf, const double *c)
{
	const int nx = p.nx, ny = p.ny;
	auto il = [nx](int ix, int iy) { return iy * nx + ix; };
	//  the start concentration (zero for the film's rows, which take none)
	auto cc = [&](int ix, int iy) { return c ? c[(size_t)il(ix, iy)] : 0.0; };
	for(int jy = 2; jy < ny - 2; ++jy)
	{
		Slot m, q;
		for(int k = 0; k < 4; ++k)
		{
			m.L[k] = il(k, jy); m.opp[k] = il(nx - 1 - k, jy);
			q.L[k] = il(nx - 1 - k, jy); q.opp[k] = il(k, jy);
		}
		m.cs = m.L[0]; m.st = 1;
		q.cs = q.L[3]; q.st = 1;
		m.cb = 0.5 * (cc(1, jy) + cc(2, jy));
		q.cb = 0.5 * (cc(nx - 2, jy) + cc(nx - 3, jy));
		ApplyEdge(w, tf, p.bc[0], m);
		ApplyEdge(w, tf, p.bc[1], q);
	}
	for(int ix = 2; ix < nx - 2; ++ix)
	{
		Slot m, q;
		for(int k = 0; k < 4; ++k)
		{
			m.L[k] = il(ix, k); m.opp[k] = il(ix, ny - 1 - k);
			q.L[k] = il(ix, ny - 1 - k); q.opp[k] = il(ix, k);
		}
		m.cs = m.L[0]; m.st = nx;
		q.cs = q.L[3]; q.st = nx;
		m.cb = 0.5 * (cc(ix, 1) + cc(ix, 2));
		q.cb = 0.5 * (cc(ix, ny - 2) + cc(ix, ny - 3));
		ApplyEdge(w, tf, p.bc[2], m);
		ApplyEdge(w, tf, p.bc[3], q);
	}
	const int xm[4] = {0, 1, 2, 3}, xp[4] = {nx - 1, nx - 2, nx - 3, nx - 4};
	const int ym[4] = {0, 1, 2, 3}, yp[4] = {ny - 1, ny - 2, ny - 3, ny - 4};
	const Corner mm = MakeCorner(nx, xm, ym), mp = MakeCorner(nx, xm, yp), pm = MakeCorner(nx, xp, ym),
	             pp = MakeCorner(nx, xp, yp);
	//  ApplyCornersAll (BoundaryCondition.cpp:486-524): the corner values
	double vMM = 0, vMP = 0, vPM = 0, vPP = 0;
	if(tf == kBcFieldConc)
	{
		vMM = 0.25 * (cc(1, 1) + cc(2, 1) + cc(1, 2) + cc(2, 2));
		vPM = 0.25 * (cc(nx - 2, 1) + cc(nx - 3, 1) + cc(nx - 2, 2) + cc(nx - 3, 2));
		vMP = 0.25 * (cc(1, ny - 2) + cc(2, ny - 2) + cc(1, ny - 3) + cc(2, ny - 3));
		vPP = 0.25 * (cc(nx - 2, ny - 2) + cc(nx - 3, ny - 2) + cc(nx - 2, ny - 3) + cc(nx - 3, ny - 3));
	}
	ApplyCorner(w, tf, p.bc[0], p.bc[2], mm, pm, mp, pp, vMM);
	ApplyCorner(w, tf, p.bc[0], p.bc[3], mp, pp, mm, pm, vMP);
	ApplyCorner(w, tf, p.bc[1], p.bc[2], pm, mm, pp, mp, vPM);
	ApplyCorner(w, tf, p.bc[1], p.bc[3], pp, mp, pm, mm, vPP);
}

} // namespace

BcPlan BuildBcPlan(const yz_step_params &p, int field, const double *c)
{
	const int nx = p.nx, ny = p.ny, n = nx * ny;
	for(int e = 0; e < 4; ++e)
		if(p.bc[e] < kBcSymmetry || p.bc[e] > kBcOutlet) throw UsageError("step: unknown edge kind");
	Rows w(n);
	ApplyAll(w, p, field, c);
	BcPlan P;
	std::vector<int> loc((size_t)n, -1);
	for(int iy = 0; iy < ny; ++iy)
		for(int ix = 0; ix < nx; ++ix)
		{
			if(ix >= 2 && ix < nx - 2 && iy >= 2 && iy < ny - 2) continue;
			const int i = iy * nx + ix;
			const Row &r = w.r[(size_t)i];
			if(!r.any) throw UsageError("step: a ghost row without a condition");
			loc[(size_t)i] = (int)P.ghost.size();
			P.ghost.push_back(i);
			std::vector<int> c(1, i);
			std::vector<double> v(1, r.diag);
			c.insert(c.end(), r.col.begin(), r.col.end());
			v.insert(v.end(), r.val.begin(), r.val.end());
			const bool copy = v.size() == 2 && v[0] == 1.0 && v[1] == -1.0 && r.rhs == 0.0 && !std::signbit(r.rhs);
			P.partner.push_back(copy ? c[1] : -1);
			P.cols.push_back(c);
			P.vals.push_back(v);
			P.rhs.push_back(r.rhs);
		}
	//  a copy whose cell is itself a ghost is coupled to that ghost's row
	//  (solved with it), not a copy of a solved value
	for(size_t g = 0; g < P.ghost.size(); ++g)
	{
		if(P.partner[g] >= 0 && loc[(size_t)P.partner[g]] >= 0) P.partner[g] = -1;
		if(P.partner[g] < 0) P.simple = false;
	}
	//  SatisfyBCRows (CRS_Matrix.cpp:198-302): the sets by union-find over
	//  the rows' nonzero entries in other ghost rows
	const int nr = (int)P.ghost.size();
	std::vector<int> parent((size_t)nr);
	for(int a = 0; a < nr; ++a) parent[(size_t)a] = a;
	auto find = [&parent](int a) {
		while(parent[(size_t)a] != a) { parent[(size_t)a] = parent[(size_t)parent[(size_t)a]]; a = parent[(size_t)a]; }
		return a;
	};
	for(int r = 0; r < nr; ++r)
		for(size_t k = 1; k < P.cols[(size_t)r].size(); ++k)
		{
			const int j = loc[(size_t)P.cols[(size_t)r][k]];
			if(j < 0 || P.vals[(size_t)r][k] == 0.0) continue;
			const int a = find(r), b = find(j);
			if(a != b) parent[(size_t)std::max(a, b)] = std::min(a, b);
		}
	std::vector<std::vector<int>> sets((size_t)nr);
	for(int r = 0; r < nr; ++r) sets[(size_t)find(r)].push_back(r);
	P.termOff.push_back(0);
	for(int c = 0; c < nr; ++c)
	{
		const std::vector<int> &set = sets[(size_t)c];
		const int m = (int)set.size();
		if(m == 0) continue;
		if(m > kMaxBcSet) throw UsageError("step: a set of more than 8 coupled ghost rows");
		std::vector<double> M((size_t)m * m, 0.0);
		std::vector<std::vector<int>> tc((size_t)m);
		std::vector<std::vector<double>> tv((size_t)m);
		bool solvable = true;
		for(int q = 0; q < m && solvable; ++q)
		{
			const std::vector<int> &cl = P.cols[(size_t)set[(size_t)q]];
			const std::vector<double> &vl = P.vals[(size_t)set[(size_t)q]];
			if(vl[0] == 0.0) { solvable = false; break; }
			std::vector<char> used(cl.size(), 0);
			for(size_t k = 0; k < cl.size(); ++k)
			{
				const int j = loc[(size_t)cl[k]];
				if(j >= 0 && find(j) == c)
				{
					const int pos = (int)(std::find(set.begin(), set.end(), j) - set.begin());
					M[(size_t)q * m + pos] += vl[k];
					used[k] = 1;
				}
			}
			//  the other terms in order of decreasing |a_ij|, ties in storage order
			for(;;)
			{
				int kb = -1;
				for(size_t k = 0; k < cl.size(); ++k)
					if(!used[k] && (kb < 0 || std::fabs(vl[k]) > std::fabs(vl[(size_t)kb]))) kb = (int)k;
				if(kb < 0) break;
				used[(size_t)kb] = 1;
				tc[(size_t)q].push_back(cl[(size_t)kb]);
				tv[(size_t)q].push_back(vl[(size_t)kb]);
			}
		}
		std::vector<int> piv((size_t)m, 0);
		std::vector<double> fac((size_t)m * m, 0.0);
		for(int col = 0; col < m && solvable; ++col)
		{
			int pv = col;
			for(int q = col + 1; q < m; ++q)
				if(std::fabs(M[(size_t)q * m + col]) > std::fabs(M[(size_t)pv * m + col])) pv = q;
			if(M[(size_t)pv * m + col] == 0.0) { solvable = false; break; }
			piv[(size_t)col] = pv;
			if(pv != col)
				for(int q = 0; q < m; ++q) std::swap(M[(size_t)pv * m + q], M[(size_t)col * m + q]);
			for(int q = col + 1; q < m; ++q)
			{
				const double f = M[(size_t)q * m + col] / M[(size_t)col * m + col];
				fac[(size_t)q * m + col] = f;
				if(f == 0.0) continue;
				for(int r = col; r < m; ++r) M[(size_t)q * m + r] -= f * M[(size_t)col * m + r];
			}
		}
		P.setM.push_back(solvable ? m : 0);
		P.setRowOff.push_back((int)P.row.size());
		P.setMatOff.push_back((int)P.U.size());
		for(int q = 0; q < m; ++q)
		{
			P.row.push_back(P.ghost[(size_t)set[(size_t)q]]);
			P.rowRhs.push_back(P.rhs[(size_t)set[(size_t)q]]);
			P.piv.push_back(piv[(size_t)q]);
			P.termCol.insert(P.termCol.end(), tc[(size_t)q].begin(), tc[(size_t)q].end());
			P.termVal.insert(P.termVal.end(), tv[(size_t)q].begin(), tv[(size_t)q].end());
			P.termOff.push_back((int)P.termCol.size());
		}
		P.fac.insert(P.fac.end(), fac.begin(), fac.end());
		P.U.insert(P.U.end(), M.begin(), M.end());
	}
	return P;
}

} // namespace yz
