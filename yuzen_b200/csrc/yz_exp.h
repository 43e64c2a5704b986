// yz_exp.h -- a correctly rounded exp(x) for double, on the host and the
// device alike (the same operations in the same order: the result is the same
// bits on both).
//
// The ConcZ step evaluates the reference's property laws, base *
// exp(k (c - c0)) (FluidProperty.h:176-180), millions of times a step, and
// the film's capillary system at the workload's size is conditioned so that
// a last-bit difference in one viscosity moves its converged answer by about
// 1e-9.  A libm's exp is faithful, not correctly rounded (the host's misrounds
// about one argument in 1,300 on [-12, 12]), and two libms misround different
// arguments; a correctly rounded exp is one function.  The oracle of the
// ConcZ model links this one in place of the libm's (oracle/probe/
// exp_shim.cpp), so that the reference's numerics and the device's are the
// same to the bit.
//
// Method (double-double arithmetic after Dekker 1971 and Knuth's TwoSum):
//   x = k ln2 + r, k = nearest integer to x / ln2, r formed in double-double
//       with ln2 split into three doubles (L1 + L2 + L3, 160 bits);
//   exp(r) = (exp(r / 256))^256, exp(r / 256) by its Taylor series to the
//       ninth power in double-double (|r / 256| <= 0.00136: the first term
//       left out is below 2^-110), then eight double-double squarings;
//   the double-double result rounded once to double and scaled by 2^k.
// The result's relative error before that one rounding is below 2^-97, so
// it is the correctly rounded exp(x) unless exp(x) lies within 2^-97 of a
// rounding boundary (for no double x in the range the library uses).
// Results below the normal range (x < -708) come from exp2(x / ln 2), with
// no claim to the bit: their scaling would round a second time, and no
// property law of the library reaches them.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define YZ_HD __host__ __device__ __forceinline__
#else
#define YZ_HD inline
#endif

namespace yz {
namespace crexp {

YZ_HD double Fma(double a, double b, double c)
{
#if defined(__CUDA_ARCH__)
	return __fma_rn(a, b, c);
#else
	return std::fma(a, b, c);
#endif
}

struct DD
{
	double hi, lo;
};

//  a + b exactly, |a| >= |b| not needed (Knuth)
YZ_HD DD TwoSum(double a, double b)
{
	const double s = a + b;
	const double bb = s - a;
	const double e = (a - (s - bb)) + (b - bb);
	return DD{s, e};
}

//  a + b exactly when |a| >= |b|
YZ_HD DD FastTwoSum(double a, double b)
{
	const double s = a + b;
	const double e = b - (s - a);
	return DD{s, e};
}

//  a * b exactly (the fused multiply-add gives the product's rounding error)
YZ_HD DD TwoProd(double a, double b)
{
	const double p = a * b;
	const double e = Fma(a, b, -p);
	return DD{p, e};
}

YZ_HD DD Add(DD a, DD b)
{
	DD s = TwoSum(a.hi, b.hi);
	const double t = a.lo + b.lo;
	s.lo = s.lo + t;
	return FastTwoSum(s.hi, s.lo);
}

YZ_HD DD Mul(DD a, DD b)
{
	DD p = TwoProd(a.hi, b.hi);
	const double t = a.hi * b.lo + a.lo * b.hi;
	p.lo = p.lo + t;
	return FastTwoSum(p.hi, p.lo);
}

YZ_HD double Exp(double x)
{
	if(!(x == x)) return x;
	if(x > 709.8) return HUGE_VAL;
	if(x < -708.0) return exp2(x * 0x1.71547652b82fep+0);
	//  ln2 = L1 + L2 + L3 and 1 / ln2, from a 80-digit ln 2
	const double L1 = 0x1.62e42fefa39efp-1, L2 = 0x1.abc9e3b39803fp-56, L3 = 0x1.7b57a079a1934p-111;
	const double INV_LN2 = 0x1.71547652b82fep+0;
	const double k = rint(x * INV_LN2);
	//  r = x - k ln2 in double-double; x - k L1 is exact (Sterbenz)
	const DD p1 = TwoProd(k, L1);
	DD r = TwoSum(x - p1.hi, -p1.lo);
	const DD p2 = TwoProd(k, L2);
	r = Add(r, DD{-p2.hi, -p2.lo});
	r = Add(r, DD{-(k * L3), 0.0});
	//  r / 256, exact
	r.hi *= 0x1p-8;
	r.lo *= 0x1p-8;
	//  1/n! as double-doubles, n = 9 .. 2, for Horner's scheme
	const double ch[8] = {0x1.71de3a556c734p-19, 0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-13,
	                      0x1.6c16c16c16c17p-10, 0x1.1111111111111p-7,  0x1.5555555555555p-5,
	                      0x1.5555555555555p-3,  0x1.0000000000000p-1};
	const double cl[8] = {-0x1.c154f8ddc6c00p-73, 0x1.a01a01a01a01ap-76, 0x1.a01a01a01a01ap-73,
	                      -0x1.f49f49f49f49fp-65, 0x1.1111111111111p-63, 0x1.5555555555555p-59,
	                      0x1.5555555555555p-57,  0.0};
	DD e = DD{ch[0], cl[0]};
	for(int i = 1; i < 8; ++i) e = Add(Mul(e, r), DD{ch[i], cl[i]});
	e = Add(Mul(e, r), DD{1.0, 0.0});
	e = Add(Mul(e, r), DD{1.0, 0.0});
	for(int i = 0; i < 8; ++i) e = Mul(e, e);
	//  e.hi is e.hi + e.lo rounded (FastTwoSum), scaled exactly by 2^k
	return ldexp(e.hi, (int)k);
}

} // namespace crexp
} // namespace yz

#undef YZ_HD
