// Op-counting build of the C oracle (test and measurement infrastructure).
//
// dms_oracle.c is compiled a second time as C++ with this header force-included and every
// `double` replaced by `counted`, a one-member struct that performs the same IEEE operation
// and increments a per-class counter: add/sub, mul, div, sqrt and library transcendentals
// (exp, erf, log1p).  The shared elementary functions of include/dms_math.h are compiled
// through the same type, so their series count as the adds and multiplies they are.
// DMS_OPS_MARK(k) counts work units: 0 RK45 attempt, 1 accepted free step, 2 scattering,
// 3 trajectory; DMS_OPS_PHASE(k) attributes the following operations to unit k.  The counts give the algorithmic FP64 operations per unit of work that
// bench.py divides by the kernel time (roofline "achieved").
#pragma once

#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace dms_ops
{
// ops[phase][class]: phase 0 RK45 attempt, 1 free-step bookkeeping, 2 scattering and segment
// start, 3 trajectory start and end; class 0 add/sub, 1 mul, 2 div, 3 sqrt, 4 transcendental
extern uint64_t ops[4][5];
extern uint64_t units[4];
extern int phase;
}	// namespace dms_ops

struct counted
{
	double v;
	counted() = default;
	template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
	counted(T x) : v(static_cast<double>(x))
	{
	}
	explicit operator double() const { return v; }
	explicit operator float() const { return static_cast<float>(v); }
	explicit operator int() const { return static_cast<int>(v); }
	explicit operator unsigned int() const { return static_cast<unsigned int>(v); }
	explicit operator long() const { return static_cast<long>(v); }
	explicit operator unsigned long() const { return static_cast<unsigned long>(v); }
	explicit operator long long() const { return static_cast<long long>(v); }
	explicit operator unsigned long long() const { return static_cast<unsigned long long>(v); }
	counted operator-() const { return counted(-v); }
	counted& operator+=(counted o)
	{
		dms_ops::ops[dms_ops::phase][0]++;
		v += o.v;
		return *this;
	}
	counted& operator-=(counted o)
	{
		dms_ops::ops[dms_ops::phase][0]++;
		v -= o.v;
		return *this;
	}
	counted& operator*=(counted o)
	{
		dms_ops::ops[dms_ops::phase][1]++;
		v *= o.v;
		return *this;
	}
	counted& operator/=(counted o)
	{
		dms_ops::ops[dms_ops::phase][2]++;
		v /= o.v;
		return *this;
	}
};

inline counted operator+(counted a, counted b)
{
	dms_ops::ops[dms_ops::phase][0]++;
	return counted(a.v + b.v);
}
inline counted operator-(counted a, counted b)
{
	dms_ops::ops[dms_ops::phase][0]++;
	return counted(a.v - b.v);
}
inline counted operator*(counted a, counted b)
{
	dms_ops::ops[dms_ops::phase][1]++;
	return counted(a.v * b.v);
}
inline counted operator/(counted a, counted b)
{
	dms_ops::ops[dms_ops::phase][2]++;
	return counted(a.v / b.v);
}
inline bool operator<(counted a, counted b) { return a.v < b.v; }
inline bool operator>(counted a, counted b) { return a.v > b.v; }
inline bool operator<=(counted a, counted b) { return a.v <= b.v; }
inline bool operator>=(counted a, counted b) { return a.v >= b.v; }
inline bool operator==(counted a, counted b) { return a.v == b.v; }
inline bool operator!=(counted a, counted b) { return a.v != b.v; }
inline bool operator!(counted a) { return !a.v; }

inline counted sqrt(counted a)
{
	dms_ops::ops[dms_ops::phase][3]++;
	return counted(std::sqrt(a.v));
}
inline counted fabs(counted a) { return counted(std::fabs(a.v)); }
inline counted floor(counted a) { return counted(std::floor(a.v)); }
inline counted exp(counted a)
{
	dms_ops::ops[dms_ops::phase][4]++;
	return counted(std::exp(a.v));
}
inline counted erf(counted a)
{
	dms_ops::ops[dms_ops::phase][4]++;
	return counted(std::erf(a.v));
}
inline counted log1p(counted a)
{
	dms_ops::ops[dms_ops::phase][4]++;
	return counted(std::log1p(a.v));
}
inline bool isfinite(counted a) { return std::isfinite(a.v); }
inline counted strtod_counted(const char* s, char** e) { return counted(std::strtod(s, e)); }

#define DMS_OPS_MARK(kind) (dms_ops::units[(kind)]++)
#define DMS_OPS_PHASE(p) (dms_ops::phase = (p))
#define double counted
