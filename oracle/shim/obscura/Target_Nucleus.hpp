// Oracle test shim: nuclear targets.  Isotope mass = m_proton for A = 1, else A * u.
// Get_Nucleus(Z) returns the stable isotopes of element Z with their natural abundances
// (IUPAC representative isotopic compositions), covering Z = 1..28 as used by the solar model.
#ifndef DMS_SHIM_TARGET_NUCLEUS_HPP
#define DMS_SHIM_TARGET_NUCLEUS_HPP
#include <string>
#include <vector>
namespace obscura
{
struct Isotope
{
	unsigned int Z = 1, A = 1;
	double abundance = 1.0;
	double spin = 0.0, sp = 0.0, sn = 0.0;
	double mass = 0.0;
	std::string name;
	Isotope() {}
	Isotope(unsigned int z, unsigned int a, double abund = 1.0);
	void Print_Summary(unsigned int MPI_rank = 0) const;
	double Helm_Form_Factor(double) const { return 1.0; }  // low-mass mode: never used
};
struct Nucleus
{
	unsigned int Z = 1;
	std::string name;
	std::vector<Isotope> isotopes;
};
void Import_Nuclear_Data();
Isotope Get_Isotope(unsigned int Z, unsigned int A);
Nucleus Get_Nucleus(unsigned int Z);
}	// namespace obscura
#endif
