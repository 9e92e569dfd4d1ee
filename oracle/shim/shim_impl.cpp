// Oracle test shim implementation: the third-party functions (libphysica, obscura, MPI) that
// the reference's own hot-path sources call, restated so those sources compile and run in
// this container without the libraries.  Test infrastructure only: built into oracle/_ref/
// together with the reference translation units, never linked into the engine.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "libphysica/Integration.hpp"
#include "libphysica/Linear_Algebra.hpp"
#include "libphysica/Natural_Units.hpp"
#include "libphysica/Numerics.hpp"
#include "libphysica/Statistics.hpp"
#include "libphysica/Utilities.hpp"
#include "mpi.h"
#include "obscura/Astronomy.hpp"
#include "obscura/DM_Halo_Models.hpp"
#include "obscura/DM_Particle_Standard.hpp"
#include "obscura/Target_Nucleus.hpp"

#include "../../include/dms_nuclear_data.h"
#include "../../include/dms_philox.h"
#include "shim_control.h"

using namespace libphysica::natural_units;

// ------------------------------------------------------------------------------------------
// Draw stream control (see shim_control.h)
namespace
{
struct DrawContext
{
	uint32_t seed = 1;
	uint32_t point = 0;
	uint64_t trajectory = 0;
	uint64_t index = 0;
	int tracing = 0;
	std::vector<double> trace;   // per scatter: r [natural], v [natural], draw index before the angle draw
};
DrawContext g_draws;
std::vector<double> g_last_knots;

double Next_Uniform()
{
	return dms_draw_uniform(g_draws.seed, g_draws.point, g_draws.trajectory, g_draws.index++);
}

void Record_Scatter(double r, double v)
{
	if(!g_draws.tracing)
		return;
	g_draws.trace.push_back(r);
	g_draws.trace.push_back(v);
	g_draws.trace.push_back(static_cast<double>(g_draws.index));
}
}	// namespace

extern "C" void dms_shim_set_stream(uint32_t seed, uint32_t point, uint64_t trajectory)
{
	g_draws.seed = seed;
	g_draws.point = point;
	g_draws.trajectory = trajectory;
	g_draws.index = 0;
	g_draws.trace.clear();
}
extern "C" uint64_t dms_shim_draw_count(void) { return g_draws.index; }
extern "C" void dms_shim_set_tracing(int on) { g_draws.tracing = on; }
extern "C" size_t dms_shim_trace_size(void) { return g_draws.trace.size(); }
extern "C" const double* dms_shim_trace_data(void) { return g_draws.trace.data(); }

// ------------------------------------------------------------------------------------------
// libphysica
namespace libphysica
{
namespace natural_units
{
std::vector<double> In_Units(const std::vector<double>& quantity, double unit)
{
	std::vector<double> r(quantity);
	for(auto& x : r) x /= unit;
	return r;
}
Vector In_Units(const Vector& quantity, double unit) { return quantity / unit; }
}	// namespace natural_units

Vector Spherical_Coordinates(double r, double theta, double phi, const Vector& axis)
{
	const Vector e3 = axis / axis.Norm();
	const Vector reference = (std::fabs(e3[2]) < 0.9) ? Vector({0.0, 0.0, 1.0}) : Vector({1.0, 0.0, 0.0});
	const Vector e1 = reference.Cross(e3).Normalized();
	const Vector e2 = e3.Cross(e1).Normalized();
	const double st = std::sin(theta), ct = std::cos(theta), cp = std::cos(phi), sp = std::sin(phi);
	Vector out(3);
	for(unsigned int i = 0; i < 3; i++)
		out[i] = r * (st * cp * e1[i] + st * sp * e2[i] + ct * e3[i]);
	return out;
}

Interpolation::Interpolation(const std::vector<std::vector<double>>& table, double dim1, double dim2)
{
	const double ux = (dim1 > 0.0) ? dim1 : 1.0;
	const double uy = (dim2 > 0.0) ? dim2 : 1.0;
	for(const auto& row : table)
	{
		xs.push_back(row[0] * ux);
		ys.push_back(row[1] * uy);
	}
	if(xs.size() < 2)
		throw std::invalid_argument("Interpolation: at least two knots are required");
	Compute_Slopes();
	g_last_knots = xs;
}

void Interpolation::Compute_Slopes()
{
	slopes.assign(xs.size() - 1, 0.0);
	for(size_t i = 0; i + 1 < xs.size(); i++)
		slopes[i] = (ys[i + 1] - ys[i]) / (xs[i + 1] - xs[i]);
}

double Interpolation::operator()(double x) const
{
	// largest i with xs[i] <= x, clamped to [0, N-2]
	size_t lo = 0, hi = xs.size() - 1;
	if(x >= xs[hi - 1])
		lo = hi - 1;
	else
	{
		while(hi - lo > 1)
		{
			const size_t mid = (lo + hi) / 2;
			if(xs[mid] <= x)
				lo = mid;
			else
				hi = mid;
		}
	}
	return ys[lo] + (x - xs[lo]) * slopes[lo];
}

void Interpolation::Multiply(double factor)
{
	for(auto& y : ys) y *= factor;
	Compute_Slopes();
}

double Integrate(std::function<double(double)> func, double a, double b, const std::string&)
{
	std::vector<double> cuts = {a};
	for(const double k : g_last_knots)
		if(k > a && k < b)
			cuts.push_back(k);
	cuts.push_back(b);
	double sum = 0.0;
	for(size_t i = 0; i + 1 < cuts.size(); i++)
	{
		const double lo = cuts[i], hi = cuts[i + 1];
		const double f_lo = func(lo), f_hi = func(hi);
		if(lo == 0.0)
		{
			sum += 0.5 * (hi - lo) * (f_lo + f_hi);
			continue;
		}
		const double g_lo = f_lo * lo * lo, g_hi = f_hi * hi * hi;
		const double h = hi - lo;
		const double s = (g_hi - g_lo) / h;
		sum += g_lo * h / (lo * hi) + s * (std::log1p(h / lo) - h / hi);
	}
	return sum;
}

double Sample_Uniform(std::mt19937&, double x_min, double x_max)
{
	const double u = Next_Uniform();
	return x_min + u * (x_max - x_min);
}

double Rejection_Sampling(const std::function<double(double)>& PDF, double xMin, double xMax, double yMax, std::mt19937& PRNG)
{
	while(true)
	{
		const double x = Sample_Uniform(PRNG, xMin, xMax);
		const double y = Sample_Uniform(PRNG, 0.0, yMax);
		if(y <= PDF(x))
			return x;
	}
}

std::vector<std::vector<double>> Import_Table(const std::string& file_path, std::vector<double> units, unsigned int lines_to_skip)
{
	std::string path = file_path;
	const char* override_path = std::getenv("DMS_SOLAR_MODEL_PATH");
	if(override_path != nullptr && path.size() >= 16 && path.compare(path.size() - 16, 16, "model_agss09.dat") == 0)
		path = override_path;
	std::ifstream in(path);
	if(!in)
		throw std::runtime_error("Import_Table: cannot open " + path);
	std::string line;
	for(unsigned int i = 0; i < lines_to_skip && std::getline(in, line); i++) {}
	std::vector<std::vector<double>> table;
	while(std::getline(in, line))
	{
		std::istringstream ss(line);
		std::vector<double> row;
		double value;
		while(ss >> value) row.push_back(value);
		if(row.empty())
			continue;
		for(size_t j = 0; j < row.size() && j < units.size(); j++) row[j] *= units[j];
		table.push_back(row);
	}
	return table;
}

std::vector<double> Linear_Space(double min, double max, unsigned int steps)
{
	std::vector<double> out(steps);
	const double step = (max - min) / (steps - 1);
	for(unsigned int i = 0; i < steps; i++) out[i] = min + i * step;
	return out;
}

std::vector<int> Range(int n)
{
	std::vector<int> out(n);
	for(int i = 0; i < n; i++) out[i] = i;
	return out;
}

double Round(double d, int digits)
{
	if(d == 0.0 || !std::isfinite(d))
		return d;
	const double scale = std::pow(10.0, digits - 1 - std::floor(std::log10(std::fabs(d))));
	return std::round(d * scale) / scale;
}

void Print_Progress_Bar(double, unsigned int, unsigned int, double) {}

std::string Time_Display(double seconds)
{
	std::ostringstream os;
	os << seconds << " s";
	return os.str();
}
}	// namespace libphysica

// ------------------------------------------------------------------------------------------
// obscura
namespace obscura
{
Isotope::Isotope(unsigned int z, unsigned int a, double abund) : Z(z), A(a), abundance(abund)
{
	mass = (A == 1) ? mProton : A * mNucleon;
}

void Isotope::Print_Summary(unsigned int) const
{
	std::cout << Z << "\t" << A << "\t" << 100.0 * abundance << std::endl;
}

void Import_Nuclear_Data() {}

Isotope Get_Isotope(unsigned int Z, unsigned int A)
{
	for(const auto& t : DMS_TARGET_ISOTOPES)
		if(t.Z == Z && t.A == A)
			return Isotope(Z, A, 1.0);
	throw std::invalid_argument("Get_Isotope: isotope not in the shim table");
}

Nucleus Get_Nucleus(unsigned int Z)
{
	Nucleus n;
	n.Z = Z;
	for(int k = 10; k < DMS_NUM_TARGETS; k++)
		if(DMS_TARGET_ISOTOPES[k].Z == Z)
			n.isotopes.push_back(Isotope(Z, DMS_TARGET_ISOTOPES[k].A, DMS_TARGET_ISOTOPES[k].abundance));
	if(n.isotopes.empty())
		throw std::invalid_argument("Get_Nucleus: element not in the shim table");
	return n;
}

double DM_Particle_SI::Sigma_Total_Nucleus(const Isotope& target, double, double)
{
	const double mu_N = mass * target.mass / (mass + target.mass);
	const double mu_p = mass * mProton / (mass + mProton);
	const double coupling = target.Z + fn_over_fp * (target.A - target.Z);
	const double ratio = mu_N / mu_p;
	return sigma_proton * ratio * ratio * coupling * coupling;
}

double DM_Particle_SI::Sigma_Total_Electron(double, double) { return sigma_electron; }

double DM_Particle::High_Mass_Not_Shimmed()
{
	throw std::logic_error("the oracle shim provides obscura's low-mass mode only");
}

double DM_Particle_SI::Sample_Scattering_Angle_Nucleus(std::mt19937& PRNG, const Isotope&, double vDM, double r)
{
	Record_Scatter(r, vDM);
	return libphysica::Sample_Uniform(PRNG, -1.0, 1.0);
}

double DM_Particle_SI::Sample_Scattering_Angle_Electron(std::mt19937& PRNG, double vDM, double r)
{
	Record_Scatter(r, vDM);
	return libphysica::Sample_Uniform(PRNG, -1.0, 1.0);
}

namespace
{
const double SQRT_PI = std::sqrt(3.14159265358979323846);
constexpr double PI_1_5 = 5.5683279968317078453;
const double GL7_X[7] = {0.0, -0.4058451513773971669066064, 0.4058451513773971669066064, -0.7415311855993944398638648, 0.7415311855993944398638648, -0.9491079123427585245261897, 0.9491079123427585245261897};
const double GL7_W[7] = {0.4179591836734693877551020, 0.3818300505051189449503698, 0.3818300505051189449503698, 0.2797053914892766679014678, 0.2797053914892766679014678, 0.1294849661688696932706114, 0.1294849661688696932706114};

template <class F>
double Composite_GL7(F f, double a, double b, int panels)
{
	const double h = (b - a) / panels;
	double sum = 0.0;
	for(int p = 0; p < panels; p++)
	{
		const double lo = a + p * h;
		const double mid = lo + 0.5 * h;
		double panel = 0.0;
		for(int k = 0; k < 7; k++) panel += GL7_W[k] * f(mid + 0.5 * h * GL7_X[k]);
		sum += 0.5 * h * panel;
	}
	return sum;
}
}	// namespace

Standard_Halo_Model::Standard_Halo_Model(double v0, double vesc, const libphysica::Vector& vobs)
: v_0(v0), v_esc(vesc), v_obs(vobs.Norm()), vel_observer(vobs)
{
	const double z = v_esc / v_0;
	N_esc = std::erf(z) - 2.0 * z * std::exp(-z * z) / SQRT_PI;
}

double Standard_Halo_Model::PDF_Velocity(const libphysica::Vector& vel)
{
	const libphysica::Vector w = vel + vel_observer;
	const double w2 = w.Dot(w);
	if(w2 > v_esc * v_esc)
		return 0.0;
	return std::exp(-w2 / (v_0 * v_0)) / (N_esc * PI_1_5 * v_0 * v_0 * v_0);
}

double Standard_Halo_Model::PDF_Speed(double v)
{
	if(v < 0.0 || v > v_esc + v_obs)
		return 0.0;
	const double dm = v - v_obs;
	const double dp = v + v_obs;
	const double a = std::exp(-dm * dm / (v_0 * v_0));
	const double b = (dp <= v_esc) ? std::exp(-dp * dp / (v_0 * v_0)) : std::exp(-v_esc * v_esc / (v_0 * v_0));
	return v / (N_esc * SQRT_PI * v_0 * v_obs) * (a - b);
}

double Standard_Halo_Model::Average_Speed(double)
{
	auto f = [this](double v) { return v * PDF_Speed(v); };
	return Composite_GL7(f, 0.0, v_esc - v_obs, 256) + Composite_GL7(f, v_esc - v_obs, v_esc + v_obs, 256);
}

double Standard_Halo_Model::Eta_Function(double)
{
	auto f = [this](double v) { return (v > 0.0) ? PDF_Speed(v) / v : 0.0; };
	return Composite_GL7(f, 0.0, v_esc - v_obs, 256) + Composite_GL7(f, v_esc - v_obs, v_esc + v_obs, 256);
}

libphysica::Vector Sun_Velocity() { return libphysica::Vector({11.1 * km / sec, 232.2 * km / sec, 7.3 * km / sec}); }
}	// namespace obscura

// ------------------------------------------------------------------------------------------
// single-rank MPI
namespace
{
size_t Type_Size(MPI_Datatype t)
{
	switch(t)
	{
		case MPI_BYTE: return 1;
		case MPI_INT:
		case MPI_UNSIGNED: return 4;
		default: return 8;
	}
}
}	// namespace
extern "C" {
int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int, int* provided)
{
	*provided = MPI_THREAD_FUNNELED;
	return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* size)
{
	*size = 1;
	return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* rank)
{
	*rank = 0;
	return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Query_thread(int* level)
{
	*level = MPI_THREAD_FUNNELED;
	return MPI_SUCCESS;
}
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
	if(send != MPI_IN_PLACE && count > 0)
		std::memcpy(recv, send, count * Type_Size(t));
	return MPI_SUCCESS;
}
int MPI_Allgather(const void* send, int count, MPI_Datatype t, void* recv, int, MPI_Datatype, MPI_Comm)
{
	if(send != MPI_IN_PLACE && count > 0)
		std::memcpy(recv, send, count * Type_Size(t));
	return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* send, int count, MPI_Datatype t, void* recv, const int*, const int* displs, MPI_Datatype, MPI_Comm)
{
	if(send != MPI_IN_PLACE && count > 0)
		std::memcpy(static_cast<char*>(recv) + displs[0] * Type_Size(t), send, count * Type_Size(t));
	return MPI_SUCCESS;
}
int MPI_Gather(const void* send, int count, MPI_Datatype t, void* recv, int, MPI_Datatype, int, MPI_Comm)
{
	if(send != MPI_IN_PLACE && send != nullptr && recv != nullptr && count > 0)
		std::memcpy(recv, send, count * Type_Size(t));
	return MPI_SUCCESS;
}
int MPI_Gatherv(const void* send, int count, MPI_Datatype t, void* recv, const int*, const int* displs, MPI_Datatype, int, MPI_Comm)
{
	if(send != MPI_IN_PLACE && send != nullptr && recv != nullptr && count > 0)
		std::memcpy(static_cast<char*>(recv) + displs[0] * Type_Size(t), send, count * Type_Size(t));
	return MPI_SUCCESS;
}
int MPI_Ibarrier(MPI_Comm, MPI_Request* r)
{
	*r = 0;
	return MPI_SUCCESS;
}
int MPI_Test(MPI_Request*, int* flag, MPI_Status*)
{
	*flag = 1;
	return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
}
