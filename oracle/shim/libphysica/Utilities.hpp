// Oracle test shim: table import, ranges and console helpers.
#ifndef DMS_SHIM_UTILITIES_HPP
#define DMS_SHIM_UTILITIES_HPP
#include <string>
#include <vector>
#include "Numerics.hpp"
#define SEPARATOR "\n----------------------------------------\n"
#define SEPARATOR_LINE "\n----------------------------------------\n"
namespace libphysica
{
// Reads whitespace-separated numeric rows after skipping `lines_to_skip` lines; column j is
// multiplied by units[j].
std::vector<std::vector<double>> Import_Table(const std::string& file_path, std::vector<double> units = {}, unsigned int lines_to_skip = 0);
std::vector<double> Linear_Space(double min, double max, unsigned int steps);
std::vector<int> Range(int n);
double Round(double d, int digits = 3);
void Print_Progress_Bar(double progress, unsigned int MPI_rank = 0, unsigned int bar_length = 50, double time = 0.0);
std::string Time_Display(double seconds);
}	// namespace libphysica
#endif
