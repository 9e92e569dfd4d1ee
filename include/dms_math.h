/*
 * dms_math.h — elementary functions shared bit-for-bit by the CUDA engine and the CPU oracle.
 *
 * Why: the trajectory algorithm has knife-edge decisions (a step that lands exactly on the
 * solar surface versus one ulp outside selects a different step-size branch,
 * src/Simulation_Trajectory.cpp:886-899), so two implementations agree trajectory-by-trajectory
 * only if every operation that feeds the state rounds identically.  IEEE +, -, *, / and sqrt
 * do (with FMA contraction disabled); library sin/cos/log/acos differ between glibc and CUDA in
 * the last bit.  These functions are written from the textbook series below, use only IEEE
 * operations in a fixed order, and therefore return the same bits on the host and the device.
 * Accuracy is about 1 ulp.
 *
 *   log:  x = m 2^e, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s = (m-1)/(m+1), Taylor
 *         series of atanh; e*ln2 added with a two-part ln2 (Cody & Waite).
 *   sin/cos: reduction by a three-part pi/2 (Cody & Waite), Taylor series on [-pi/4, pi/4].
 *   acos: pi/2 - asin(x) for |x| <= 1/2, else 2 asin(sqrt((1 -+ x)/2)); Taylor series of asin.
 *   pow(x, 1/4) is sqrt(sqrt(x)); pow(c, 2) is c*c (exact: the correctly rounded square).
 * The split constants are the leading bits of pi/2 and ln 2 (computed from their decimal
 * expansions), chosen so that k*PIO2_1, k*PIO2_2 and e*LN2_HI are exact.
 */
#ifndef DMS_MATH_H
#define DMS_MATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define DMS_MATH_FN __host__ __device__ __forceinline__
#include <math.h>
#else
#define DMS_MATH_FN static inline
#include <math.h>
#include <string.h>
#endif

#define DMS_PI 3.141592653589793
#define DMS_PIO2_1 0x1.921fb54800000p+0
#define DMS_PIO2_2 (-0x1.de973dc800000p-31)
#define DMS_PIO2_3 (-0x1.9d9cceba3f91fp-62)
#define DMS_TWO_OVER_PI 0.6366197723675814
#define DMS_LN2_HI 0x1.62e42ff000000p-1
#define DMS_LN2_LO (-0x1.718432a1b0e26p-35)

DMS_MATH_FN uint64_t dms_bits(double x)
{
#if defined(__CUDA_ARCH__)
	return (uint64_t)__double_as_longlong(x);
#else
	uint64_t u;
	memcpy(&u, &x, sizeof u);
	return u;
#endif
}

DMS_MATH_FN double dms_from_bits(uint64_t u)
{
#if defined(__CUDA_ARCH__)
	return __longlong_as_double((long long)u);
#else
	double x;
	memcpy(&x, &u, sizeof x);
	return x;
#endif
}

/* Natural logarithm. */
DMS_MATH_FN double dms_log(double x)
{
	if(!(x > 0.0))
		return (x == 0.0) ? -INFINITY : NAN;
	if(!(x < INFINITY))
		return x;
	int e = 0;
	if(x < 2.2250738585072014e-308) /* subnormal: scale by 2^54 */
	{
		x *= 18014398509481984.0;
		e = -54;
	}
	const uint64_t u = dms_bits(x);
	e += (int)((u >> 52) & 0x7ff) - 1023;
	double m = dms_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1, 2) */
	if(m > 1.4142135623730951)
	{
		m *= 0.5;
		e += 1;
	}
	const double s = (m - 1.0) / (m + 1.0);
	const double z = s * s;
	double p = 1.0 / 23.0;
	p = p * z + 1.0 / 21.0;
	p = p * z + 1.0 / 19.0;
	p = p * z + 1.0 / 17.0;
	p = p * z + 1.0 / 15.0;
	p = p * z + 1.0 / 13.0;
	p = p * z + 1.0 / 11.0;
	p = p * z + 1.0 / 9.0;
	p = p * z + 1.0 / 7.0;
	p = p * z + 1.0 / 5.0;
	p = p * z + 1.0 / 3.0;
	const double two_s = 2.0 * s;
	const double ed = (double)e;
	return ed * DMS_LN2_HI + (two_s + (two_s * z * p + ed * DMS_LN2_LO));
}

/* sin and cos of the reduced argument r in [-pi/4, pi/4]. */
DMS_MATH_FN double dms_sin_kernel(double r)
{
	const double z = r * r;
	double p = -1.0 / 121645100408832000.0;          /* -1/19! */
	p = p * z + 1.0 / 355687428096000.0;             /*  1/17! */
	p = p * z - 1.0 / 1307674368000.0;               /* -1/15! */
	p = p * z + 1.0 / 6227020800.0;                  /*  1/13! */
	p = p * z - 1.0 / 39916800.0;                    /* -1/11! */
	p = p * z + 1.0 / 362880.0;                      /*  1/9!  */
	p = p * z - 1.0 / 5040.0;                        /* -1/7!  */
	p = p * z + 1.0 / 120.0;                         /*  1/5!  */
	p = p * z - 1.0 / 6.0;                           /* -1/3!  */
	return r + r * z * p;
}

DMS_MATH_FN double dms_cos_kernel(double r)
{
	const double z = r * r;
	double p = 1.0 / 6402373705728000.0;             /*  1/18! */
	p = p * z - 1.0 / 20922789888000.0;              /* -1/16! */
	p = p * z + 1.0 / 87178291200.0;                 /*  1/14! */
	p = p * z - 1.0 / 479001600.0;                   /* -1/12! */
	p = p * z + 1.0 / 3628800.0;                     /*  1/10! */
	p = p * z - 1.0 / 40320.0;                       /* -1/8!  */
	p = p * z + 1.0 / 720.0;                         /*  1/6!  */
	p = p * z - 1.0 / 24.0;                          /* -1/4!  */
	const double half_z = 0.5 * z;
	return 1.0 - (half_z + z * z * p);
}

/* sin and cos together; |x| up to ~1e6 (reduction exact for |k| < 2^22). */
DMS_MATH_FN void dms_sincos(double x, double* s, double* c)
{
	if(!(x - x == 0.0)) /* inf or nan */
	{
		*s = NAN;
		*c = NAN;
		return;
	}
	const double k = floor(x * DMS_TWO_OVER_PI + 0.5);
	const double r = ((x - k * DMS_PIO2_1) - k * DMS_PIO2_2) - k * DMS_PIO2_3;
	const double sr = dms_sin_kernel(r);
	const double cr = dms_cos_kernel(r);
	const long long q = ((long long)k) & 3;
	if(q == 0)
	{
		*s = sr;
		*c = cr;
	}
	else if(q == 1)
	{
		*s = cr;
		*c = -sr;
	}
	else if(q == 2)
	{
		*s = -sr;
		*c = -cr;
	}
	else
	{
		*s = -cr;
		*c = sr;
	}
}

DMS_MATH_FN double dms_sin(double x)
{
	double s, c;
	dms_sincos(x, &s, &c);
	return s;
}

DMS_MATH_FN double dms_cos(double x)
{
	double s, c;
	dms_sincos(x, &s, &c);
	return c;
}

/* asin(t) for |t| <= 1/2 by its Taylor series; term ratio (2n-1)^2 / ((2n)(2n+1)) t^2. */
DMS_MATH_FN double dms_asin_small(double t)
{
	const double z = t * t;
	double term = t;
	double sum = 0.0;
	for(int n = 1; n <= 30; n++)
	{
		const double a = (double)(2 * n - 1);
		term = term * z * (a * a) / ((double)(2 * n) * (double)(2 * n + 1));
		sum += term;
	}
	return t + sum;
}

DMS_MATH_FN double dms_acos(double x)
{
	if(!(x >= -1.0 && x <= 1.0))
		return NAN;
	if(x <= 0.5 && x >= -0.5)
		return 0.5 * DMS_PI - dms_asin_small(x);
	if(x > 0.5)
		return 2.0 * dms_asin_small(sqrt((1.0 - x) * 0.5));
	return DMS_PI - 2.0 * dms_asin_small(sqrt((1.0 + x) * 0.5));
}

/* pow(x, 0.25) of the RK45 step controller, src/Simulation_Trajectory.cpp:495 */
DMS_MATH_FN double dms_pow_quarter(double x) { return sqrt(sqrt(x)); }

#endif /* DMS_MATH_H */
