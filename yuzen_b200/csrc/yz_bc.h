// yz_bc.h -- the ghost rows of the film-height system, written on the host
// once per step context: their pattern, the Newton matrix's values on them,
// and the programme that satisfies them exactly after each solve.
//
// BoundaryCondition2D::Apply (BoundaryCondition.cpp:104-187, 376-517) writes
// the rows of the two ghost layers of every edge and the four ghost rows of
// every corner: Symmetry and Periodic copy a cell (EqualVal), Pinning holds
// the film at zero on the wall face with no tangential velocity, FreshInlet
// holds the film at its start value (Dirichlet, the third difference zero),
// Outlet sets the second and third differences to zero; the corners mirror,
// copy or take the reference's five-point stencils.  The reference applies
// it once with the film's values to A (which fixes the pattern: the diagonal
// first, the other columns in the order written) and once with the
// correction's (HeightJacobi) to the Jacobian; the Newton matrix's ghost rows
// are the latter, their right-hand side zero.
//
// CRS_Matrix::SatisfyBCRows (CRS_Matrix.cpp:198-302) then solves the ghost
// rows of the solution exactly: the rows are grouped into the sets that
// refer to one another's unknowns, each set's right-hand side less its terms
// in other unknowns (summed in order of decreasing |a_ij|, ties in storage
// order), and a set of more than one row solved by Gaussian elimination with
// partial pivoting.  The rows' values are fixed, so the host makes the
// pivoting, the multipliers and the eliminated matrix once (the same
// operations as the reference, in double), and the device kernel does the
// rest: the sums, the elimination of the right-hand side and the back
// substitution.
#pragma once

#include "yuzen_b200.h"

#include <vector>

namespace yz {

//  the reference's edge kinds (BoundaryCondition::tBoundaryCondition)
enum { kBcSymmetry = 0, kBcPeriodic = 1, kBcPinning = 2, kBcFreshInlet = 3, kBcOutlet = 4 };

struct BcPlan
{
	//  the ghost rows in ascending order, each with its columns in storage
	//  order (diagonal first), the Newton matrix's values and right-hand side
	std::vector<int> ghost;
	std::vector<std::vector<int>> cols;
	std::vector<std::vector<double>> vals;
	std::vector<double> rhs;
	//  every ghost row a copy of one cell ([1, -1], right-hand side 0): the
	//  solve's ghosts are then x[ghost] = x[partner]
	bool simple = true;
	std::vector<int> partner;
	//  SatisfyBCRows: per set its size m (0: left alone, a zero pivot),
	//  offsets into the flat arrays, rows, right-hand sides, the outside
	//  terms of each row in summation order, the pivot row of each
	//  elimination step, the multipliers (m x m, below the diagonal) and the
	//  eliminated matrix (m x m, on and above the diagonal)
	std::vector<int> setM, setRowOff, setMatOff;
	std::vector<int> row;
	std::vector<double> rowRhs;
	std::vector<int> termOff;          // per row of every set, into termCol / termVal (+1 at the end)
	std::vector<int> termCol;
	std::vector<double> termVal;
	std::vector<int> piv;              // per set row: the pivot chosen at that step
	std::vector<double> fac, U;        // m*m per set
};

constexpr int kMaxBcSet = 8;

//  a plan on the device, as the SatisfyBCRows kernel reads it; rhsVec
//  non-null: the right-hand side of row i is rhsVec[i] instead of the plan's
struct BcSets
{
	int n;
	const int *m, *rowOff, *matOff, *row, *termOff, *termCol, *piv;
	const double *rhs, *termVal, *fac, *U;
	const double *rhsVec;
};

//  the rows of the film's Newton matrix (the correction's, HeightJacobi) or
//  of the concentration equation (Conc: its values, and its right-hand side
//  from the start concentration c next to the edges and corners)
enum { kBcFieldHeight = 0, kBcFieldConc = 1 };

//  the plan of a grid with the edges of p (throws UsageError for a corner
//  the reference does not implement or leaves open); c: the start
//  concentration (n values) for the Conc field, else null
BcPlan BuildBcPlan(const yz_step_params &p, int field = kBcFieldHeight, const double *c = nullptr);

} // namespace yz
