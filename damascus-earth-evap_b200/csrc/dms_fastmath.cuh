// Correctly rounded FP64 division and square root as straight-line code, with a certificate.
//
// Why: an IEEE double division or square root compiles to a sequence with a slow-path branch.
// A lone lane of the trajectory kernel (the tail of a launch) executes a dependent chain of about
// sixty of them per RK45 step, and the branches keep the compiler from interleaving independent
// work across them.  The functions below are branch-free.  Each one also returns a certificate:
// a proof, from the exact remainder, that its result is the correctly rounded one.  When a
// certificate fails, the caller recomputes its whole unit of work (one RK45 attempt) with IEEE
// `/` and `sqrt()`, so results are always bit-identical with IEEE arithmetic.  A certificate fails
// on non-finite or subnormal operands and on results far outside the physics ranges (round to
// nearest has no ties for division and square root).
//
// Method (published, restated here from the mathematics):
//  * reciprocal and reciprocal square root: the hardware approximation (PTX rcp.approx.ftz.f64,
//    rsqrt.approx.ftz.f64) refined by Newton-Raphson iterations written with fused multiply-add
//    (P. Markstein, "IA-64 and Elementary Functions", Prentice Hall 2000, ch. 8);
//  * quotient and root: Markstein's correction step q1 = q0 + (a - b q0) y, s1 = s0 + (x - s0^2) h;
//  * certificate: q is RN(a/b) iff |a - b q| < ulp(q) |b| / 2 (strictly).  The remainder of a
//    faithful quotient is exactly representable (S. Boldo and M. Daumas, "Representable
//    correcting terms for possibly underflowing floating point operations", ARITH 16, 2003), and
//    fma computes it with at most one rounding, so the test below uses a relative margin of
//    2^-50 that covers that rounding.  s is RN(sqrt(x)) iff |x - s^2| < s ulp(s) (up to terms
//    of relative size 2^-54, covered by the same margin).  On the lower side of a power of two
//    the spacing is ulp/2; the test uses the smaller spacing, which only makes it stricter.
#pragma once

#include <cstdint>

namespace dms
{
namespace fast
{

__device__ __forceinline__ double rcp_approx(double x)
{
	double y;
	asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
	return y;
}

__device__ __forceinline__ double rsqrt_approx(double x)
{
	double y;
	asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
	return y;
}

// The smaller of the two spacings of the floating-point numbers around a positive normal q,
// scaled by `scale` (an exact power-of-two multiple), times (1 - 2^-50); 0 when q is outside
// [2^-960, 2^1000] or not finite, which makes every certificate that uses it fail.
__device__ __forceinline__ double half_spacing_times(double q, double scale)
{
	const uint64_t u = static_cast<uint64_t>(__double_as_longlong(q)) & 0x7fffffffffffffffULL;
	const int e = static_cast<int>(u >> 52);
	const int lower = (u & 0x000fffffffffffffULL) == 0 ? 1 : 0;  // a power of two: spacing below is half
	const int ue = e - 52 - 1 - lower;                            // exponent of the half spacing
	const bool in_range = e >= 63 && e <= 2023;
	const double half_ulp = __longlong_as_double(static_cast<long long>(static_cast<uint64_t>(in_range ? ue : 1) << 52));
	return in_range ? (half_ulp * scale) * (1.0 - 0x1p-50) : 0.0;
}

// 1/b to within about one ulp (not necessarily correctly rounded): two Newton-Raphson steps
// from the hardware approximation.  Shared by every quotient with divisor b.
struct Recip
{
	double b, y;
};

__device__ __forceinline__ Recip recip(double b)
{
	Recip r;
	r.b = b;
	double y = rcp_approx(b);
	double e = __fma_rn(-b, y, 1.0);
	y = __fma_rn(y, e, y);
	e = __fma_rn(-b, y, 1.0);
	r.y = __fma_rn(y, e, y);
	return r;
}

// a / b, correctly rounded when the certificate holds (ok is cleared otherwise).
__device__ __forceinline__ double div(double a, const Recip& d, bool& ok)
{
	const double q0 = __dmul_rn(a, d.y);
	const double r0 = __fma_rn(-d.b, q0, a);
	const double q1 = __fma_rn(r0, d.y, q0);
	const double r1 = __fma_rn(-d.b, q1, a);
	const double bound = half_spacing_times(q1, fabs(d.b));
	// an exact zero quotient needs a zero dividend (0/b = 0 exactly, with the sign IEEE gives)
	const bool zero_ok = (q1 == 0.0) & (a == 0.0);
	ok &= ((fabs(r1) < bound) & (fabs(a) > 0x1p-900)) | zero_ok;
	return q1;
}

__device__ __forceinline__ double div(double a, double b, bool& ok) { return div(a, recip(b), ok); }

// sqrt(x), correctly rounded when the certificate holds.
__device__ __forceinline__ double sqrt(double x, bool& ok)
{
	double y = rsqrt_approx(x);                   // ~ 1/sqrt(x)
	double h = 0.5 * y;                           // ~ 1/(2 sqrt(x))
	double s = __dmul_rn(x, y);                   // ~ sqrt(x)
	double e = __fma_rn(-s, h, 0.5);              // Goldschmidt step: s and h together
	s = __fma_rn(s, e, s);
	h = __fma_rn(h, e, h);
	e = __fma_rn(-s, h, 0.5);
	s = __fma_rn(s, e, s);
	h = __fma_rn(h, e, h);
	const double d0 = __fma_rn(-s, s, x);         // Markstein's correction
	const double s1 = __fma_rn(d0, h, s);
	const double d1 = __fma_rn(-s1, s1, x);
	const double bound = 2.0 * half_spacing_times(s1, s1);  // s ulp_min(s) (1 - 2^-50)
	// below 2^-800 the bound itself would fall into the subnormal range and round
	ok &= (fabs(d1) < bound) & (x > 0x1p-800) & (x < 0x1p+1000);
	return s1;
}

}	// namespace fast
}	// namespace dms
