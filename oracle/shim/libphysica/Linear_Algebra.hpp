// Oracle test shim: the 3-vector subset of libphysica::Vector used by the reference's
// trajectory code.  Component-wise operations in index order; Norm = sqrt(sum x_i^2);
// Normalized = v / Norm (component-wise division).  The C oracle and the CUDA engine use
// exactly these formulas.
#ifndef DMS_SHIM_LINEAR_ALGEBRA_HPP
#define DMS_SHIM_LINEAR_ALGEBRA_HPP
#include <cmath>
#include <initializer_list>
#include <ostream>
#include <vector>
#include "Natural_Units.hpp"
namespace libphysica
{
class Vector
{
	std::vector<double> components;

  public:
	Vector() : components() {}
	explicit Vector(unsigned int dim) : components(dim, 0.0) {}
	Vector(std::initializer_list<double> values) : components(values) {}
	Vector(const std::vector<double>& values) : components(values) {}
	unsigned int Size() const { return components.size(); }
	double& operator[](unsigned int i) { return components[i]; }
	const double& operator[](unsigned int i) const { return components[i]; }
	double Dot(const Vector& other) const
	{
		double sum = 0.0;
		for(unsigned int i = 0; i < components.size(); i++)
			sum += components[i] * other.components[i];
		return sum;
	}
	double Norm() const { return std::sqrt(Dot(*this)); }
	Vector Cross(const Vector& b) const
	{
		const Vector& a = *this;
		return Vector({a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]});
	}
	Vector Normalized() const;
	void Normalize() { *this = Normalized(); }
	Vector operator+(const Vector& o) const
	{
		Vector r(Size());
		for(unsigned int i = 0; i < Size(); i++) r[i] = components[i] + o[i];
		return r;
	}
	Vector operator-(const Vector& o) const
	{
		Vector r(Size());
		for(unsigned int i = 0; i < Size(); i++) r[i] = components[i] - o[i];
		return r;
	}
	Vector operator-() const
	{
		Vector r(Size());
		for(unsigned int i = 0; i < Size(); i++) r[i] = -components[i];
		return r;
	}
	Vector operator/(double s) const
	{
		Vector r(Size());
		for(unsigned int i = 0; i < Size(); i++) r[i] = components[i] / s;
		return r;
	}
	Vector& operator+=(const Vector& o) { return *this = *this + o; }
	Vector& operator-=(const Vector& o) { return *this = *this - o; }
	bool operator==(const Vector& o) const { return components == o.components; }
	friend Vector operator*(double s, const Vector& v)
	{
		Vector r(v.Size());
		for(unsigned int i = 0; i < v.Size(); i++) r[i] = s * v[i];
		return r;
	}
	friend Vector operator*(const Vector& v, double s) { return s * v; }
	friend std::ostream& operator<<(std::ostream& os, const Vector& v)
	{
		os << "(";
		for(unsigned int i = 0; i < v.Size(); i++) os << (i ? "," : "") << v[i];
		return os << ")";
	}
};
inline Vector Vector::Normalized() const { return (*this) / Norm(); }

// Vector of length r at polar angle theta from `axis` and azimuth phi about it.  Frame:
// e3 = axis/|axis|, e1 = normalize(ref x e3) with ref = z-hat unless |e3_z| >= 0.9 (then
// x-hat), e2 = normalize(e3 x e1) -- the same stable frame the reference builds in
// src/Simulation_Trajectory.cpp:109-128.
Vector Spherical_Coordinates(double r, double theta, double phi, const Vector& axis = Vector({0.0, 0.0, 1.0}));
}	// namespace libphysica
#endif
