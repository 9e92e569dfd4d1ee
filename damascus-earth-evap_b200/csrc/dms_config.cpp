// libconfig-subset parser and run-key validation; see dms_config.h.  Error texts follow the
// reference's Configuration (src/Parameter_Scan.cpp:90-471) where its tests grep for them.
#include "dms_config.h"

#include "../../include/dms.h"
#include "../../include/dms_constants.h"

#include <cctype>
#include <cmath>
#include <fstream>
#include <limits>
#include <sstream>

namespace dms
{

namespace
{
struct Lexer
{
	const std::string& s;
	size_t i = 0;
	int line = 1;
	explicit Lexer(const std::string& text) : s(text) {}

	void Skip()
	{
		for(;;)
		{
			while(i < s.size() && std::isspace(static_cast<unsigned char>(s[i])))
			{
				if(s[i] == '\n')
					line++;
				i++;
			}
			if(i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/')
			{
				while(i < s.size() && s[i] != '\n') i++;
				continue;
			}
			if(i < s.size() && s[i] == '#')
			{
				while(i < s.size() && s[i] != '\n') i++;
				continue;
			}
			if(i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*')
			{
				i += 2;
				while(i + 1 < s.size() && !(s[i] == '*' && s[i + 1] == '/'))
				{
					if(s[i] == '\n')
						line++;
					i++;
				}
				i += 2;
				continue;
			}
			return;
		}
	}
	bool Eof()
	{
		Skip();
		return i >= s.size();
	}
	char Peek()
	{
		Skip();
		return i < s.size() ? s[i] : '\0';
	}
};

std::string Error(const Lexer& L, const std::string& what) { return "configuration parse error at line " + std::to_string(L.line) + ": " + what; }

std::string Parse_Value(Lexer& L, ConfigValue& v);

std::string Parse_List(Lexer& L, ConfigValue& v, char close)
{
	v.kind = ConfigValue::List;
	L.i++;  // opening bracket
	if(L.Peek() == close)
	{
		L.i++;
		return "";
	}
	for(;;)
	{
		ConfigValue item;
		const std::string e = Parse_Value(L, item);
		if(!e.empty())
			return e;
		v.items.push_back(item);
		const char c = L.Peek();
		if(c == ',')
		{
			L.i++;
			continue;
		}
		if(c == close)
		{
			L.i++;
			return "";
		}
		return Error(L, "expected ',' or closing bracket in list");
	}
}

std::string Parse_Value(Lexer& L, ConfigValue& v)
{
	const char c = L.Peek();
	if(c == '(')
		return Parse_List(L, v, ')');
	if(c == '[')
		return Parse_List(L, v, ']');
	if(c == '"')
	{
		v.kind = ConfigValue::String;
		// adjacent string literals concatenate
		while(L.Peek() == '"')
		{
			L.i++;
			while(L.i < L.s.size() && L.s[L.i] != '"')
			{
				if(L.s[L.i] == '\\' && L.i + 1 < L.s.size())
				{
					const char e = L.s[++L.i];
					v.text += (e == 'n') ? '\n' : (e == 't') ? '\t' : e;
				}
				else
					v.text += L.s[L.i];
				L.i++;
			}
			if(L.i >= L.s.size())
				return Error(L, "unterminated string");
			L.i++;
		}
		return "";
	}
	// word: boolean or number
	const size_t start = L.i;
	while(L.i < L.s.size() && (std::isalnum(static_cast<unsigned char>(L.s[L.i])) || L.s[L.i] == '.' || L.s[L.i] == '-' || L.s[L.i] == '+' || L.s[L.i] == '_'))
		L.i++;
	std::string w = L.s.substr(start, L.i - start);
	if(w.empty())
		return Error(L, "expected a value");
	std::string lw;
	for(char ch : w) lw += static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
	if(lw == "true" || lw == "false")
	{
		v.kind = ConfigValue::Boolean;
		v.boolean = (lw == "true");
		return "";
	}
	if(lw.size() > 1 && (lw.back() == 'l'))
		w.pop_back();
	if(w.size() > 1 && (w.back() == 'L' || w.back() == 'l'))
		w.pop_back();
	v.kind = ConfigValue::Number;
	const bool hex = w.size() > 2 && w[0] == '0' && (w[1] == 'x' || w[1] == 'X');
	v.is_integer = hex || w.find_first_of(".eE") == std::string::npos;
	char* end = nullptr;
	if(hex)
		v.number = static_cast<double>(std::strtoull(w.c_str(), &end, 16));
	else
		v.number = std::strtod(w.c_str(), &end);
	if(end == nullptr || *end != '\0')
		return Error(L, "malformed number '" + w + "'");
	return "";
}
}	// namespace

std::string Parse_Config(const std::string& text, std::map<std::string, ConfigValue>& out)
{
	Lexer L(text);
	while(!L.Eof())
	{
		const size_t start = L.i;
		while(L.i < L.s.size() && (std::isalnum(static_cast<unsigned char>(L.s[L.i])) || L.s[L.i] == '_' || L.s[L.i] == '-' || L.s[L.i] == '*'))
			L.i++;
		const std::string name = L.s.substr(start, L.i - start);
		if(name.empty())
			return Error(L, "expected a setting name");
		const char sep = L.Peek();
		if(sep != '=' && sep != ':')
			return Error(L, "expected '=' after '" + name + "'");
		L.i++;
		ConfigValue v;
		const std::string e = Parse_Value(L, v);
		if(!e.empty())
			return e;
		const char end = L.Peek();
		if(end == ';' || end == ',')
			L.i++;
		out[name] = v;
	}
	return "";
}

namespace
{
struct Keys
{
	const std::map<std::string, ConfigValue>& m;
	bool Has(const char* k) const { return m.count(k) > 0; }
	const ConfigValue* Get(const char* k) const
	{
		auto it = m.find(k);
		return it == m.end() ? nullptr : &it->second;
	}
	bool Number(const char* k, double& out) const
	{
		const ConfigValue* v = Get(k);
		if(!v || v->kind != ConfigValue::Number)
			return false;
		out = v->number;
		return true;
	}
	bool Str(const char* k, std::string& out) const
	{
		const ConfigValue* v = Get(k);
		if(!v || v->kind != ConfigValue::String)
			return false;
		out = v->text;
		return true;
	}
	bool Bool(const char* k, bool& out) const
	{
		const ConfigValue* v = Get(k);
		if(!v || v->kind != ConfigValue::Boolean)
			return false;
		out = v->boolean;
		return true;
	}
};

// DM distribution: the Standard Halo Model settings
std::string Load_Halo(const Keys& k, RunConfig& cfg)
{
	std::string dist = "SHM";
	k.Str("DM_distribution", dist);
	if(dist != "SHM")
		return "Error: DM_distribution " + dist + " is not provided by this engine (SHM is).";
	k.Number("DM_local_density", cfg.rho_local);
	k.Number("SHM_v0", cfg.v0);
	k.Number("SHM_vEscape", cfg.vesc);
	if(const ConfigValue* v = k.Get("SHM_vObserver"))
	{
		if(v->kind != ConfigValue::List || v->items.size() != 3)
			return "Error: 'SHM_vObserver' must be a list of three velocities.";
		for(int i = 0; i < 3; i++) cfg.vobs[i] = v->items[i].number;
	}
	return "";
}
}	// namespace

std::string Load_Run_Config(const std::string& path, RunConfig& cfg)
{
	std::ifstream in(path);
	if(!in)
		return "Error: cannot read configuration file " + path + ".";
	std::stringstream ss;
	ss << in.rdbuf();
	std::map<std::string, ConfigValue> m;
	const std::string perr = Parse_Config(ss.str(), m);
	if(!perr.empty())
		return perr;
	Keys k{m};
	double x = 0.0;
	k.Str("ID", cfg.id);
	// Import_Parameter_Scan_Parameter, src/Parameter_Scan.cpp:90-384
	if(!k.Number("sample_size", x))
		return "No 'sample_size' setting in configuration file.";
	if(x <= 0.0)
		return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'sample_size' must be positive.";
	cfg.sample_size = static_cast<uint32_t>(x);
	if(k.Number("fixed_seed", x))
	{
		if(x < 0.0)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'fixed_seed' must be non-negative.";
		cfg.fixed_seed = static_cast<uint32_t>(x);
	}
	if(!k.Str("run_mode", cfg.run_mode))
		return "No 'run_mode' setting in configuration file.";
	cfg.capture_mode = (cfg.run_mode == "Capture");
	bool b = false;
	if(k.Bool("capture_mode", b))
		cfg.capture_mode = b;
	if(cfg.run_mode == "Capture")
		cfg.capture_mode = true;
	if(k.Number("isoreflection_rings", x))
	{
		if(x <= 0.0)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'isoreflection_rings' must be positive.";
		cfg.isoreflection_rings = static_cast<uint32_t>(x);
	}
	if(k.Number("interpolation_points", x))
	{
		if(x < 0.0)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'interpolation_points' must be non-negative.";
		cfg.interpolation_points = static_cast<uint32_t>(x);
	}
	k.Str("output_dir", cfg.output_dir);
	if(k.Number("max_trajectories", x))
	{
		if(x < 0.0)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'max_trajectories' must be non-negative.";
		cfg.max_trajectories = static_cast<uint32_t>(x);
	}
	if(k.Has("maximum_number_of_scatterings"))
	{
		if(!k.Number("maximum_number_of_scatterings", x) || !std::isfinite(x) || x < 0.0 || std::floor(x) != x || x > 1.8e19)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'maximum_number_of_scatterings' must be a non-negative integer.";
		cfg.maximum_number_of_scatterings = static_cast<uint64_t>(x);
	}
	// snapshot settings, src/Parameter_Scan.cpp:310-340
	k.Bool("snapshot_enabled", cfg.snapshot_enabled);
	if(cfg.snapshot_enabled && k.Has("snapshot_interval"))
	{
		if(!k.Number("snapshot_interval", x))
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'snapshot_interval' must be a numeric value.";
		if(!std::isfinite(x) || x < 1.0 || x > 2147483647.0 || std::floor(x) != x)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'snapshot_interval' must be a positive integer number of seconds.";
		cfg.snapshot_interval = x;
	}
	if(k.Number("max_trajectory_wall_time_sec", x))
	{
		if(!std::isfinite(x) || x < 0.0)
			return "Error in Configuration::Import_Parameter_Scan_Parameter(): 'max_trajectory_wall_time_sec' must be finite and non-negative.";
		cfg.max_trajectory_wall_time_sec = x;
	}
	if(cfg.run_mode != "Parameter point" && cfg.run_mode != "Parameter scan" && cfg.run_mode != "Custom" && cfg.run_mode != "Capture")
		return "Error in Configuration::Import_Parameter_Scan_Parameter(): Run mode " + cfg.run_mode + " not recognized.";
	if(cfg.run_mode != "Parameter point" && cfg.run_mode != "Capture")
		return "Error: run mode " + cfg.run_mode + " is not provided by this engine (Parameter point and Capture are).";

	// Construct_DM_Particle, src/Parameter_Scan.cpp:386-471
	if(!k.Number("DM_mass", cfg.DM_mass_gev))
		return "No 'DM_mass' setting in configuration file.";
	if(!k.Number("DM_spin", cfg.DM_spin))
		return "No 'DM_spin' setting in configuration file.";
	if(!k.Number("DM_fraction", cfg.DM_fraction))
		return "No 'DM_fraction' setting in configuration file.";
	if(!k.Bool("DM_light", cfg.DM_light))
		return "No 'DM_light' setting in configuration file.";
	if(!std::isfinite(cfg.DM_mass_gev) || cfg.DM_mass_gev <= 0.0 || !std::isfinite(cfg.DM_spin) || cfg.DM_spin < 0.0 ||
	   !std::isfinite(cfg.DM_fraction) || cfg.DM_fraction <= 0.0 || cfg.DM_fraction > 1.0)
		return "Error in Configuration::Construct_DM_Particle(): DM mass, spin, and fraction must be finite and physical.";
	if(!k.Str("DM_interaction", cfg.DM_interaction))
		return "No 'DM_interaction' setting in configuration file.";
	if(cfg.DM_interaction != "SI" && cfg.DM_interaction != "SD" && cfg.DM_interaction != "Dark photon")
		return "Error in DaMaSCUS_SUN::Configuration::Construct_DM_Particle(): 'DM_interaction' setting " + cfg.DM_interaction +
		       " in configuration file not recognized.";
	if(cfg.DM_interaction == "SD")
		return "Error: DM_interaction SD is not provided by this engine (SI and Dark photon are).";
	if(!cfg.DM_light)
		return "Error: DM_light = false (nuclear form factors) is not provided by this engine.";
	if(cfg.DM_interaction == "Dark photon")
	{
		// Construct_DM_Particle_Dark_Photon, src/Parameter_Scan.cpp:473-520, and the form factors
		// the dark photon accepts (src/Dark_Photon.cpp:75-88); Electric-Dipole and Long-Range stop
		// at the first rate evaluation with an IR divergence (:167-172)
		if(!k.Str("DM_form_factor", cfg.DM_form_factor))
			return "Error in DaMaSCUS_SUN::Configuration::Construct_DM_Particle_DP(): No 'DM_form_factor' setting in configuration file.";
		if(cfg.DM_form_factor == "General")
		{
			if(!k.Number("DM_mediator_mass", cfg.mediator_mass_mev))
				return "Error in Configuration::Construct_DM_Particle_DP(): No 'DM_mediator_mass' setting in configuration file.";
			if(!std::isfinite(cfg.mediator_mass_mev) || cfg.mediator_mass_mev <= 0.0)
				return "Error in Configuration::Construct_DM_Particle_DP(): 'DM_mediator_mass' must be finite and positive for the General form factor.";
			cfg.interaction = DMS_INTERACTION_DARK_PHOTON_GENERAL;
		}
		else if(cfg.DM_form_factor == "Electric-Dipole" || cfg.DM_form_factor == "Long-Range")
			return "Error in obscura::DM_Particle_Dark_Photon::Sigma_Nucleus(): Divergence in the IR.";
		else if(cfg.DM_form_factor == "Contact")
			cfg.interaction = DMS_INTERACTION_DARK_PHOTON_CONTACT;
		else
			return "Error in obscura::DM_Particle_Dark_Photon::Set_FormFactor_DM(): Form factor " + cfg.DM_form_factor + " not recognized.";
		if(!k.Number("DM_cross_section_electron", cfg.sigma_electron_cm2))
			return "Error in Configuration::Construct_DM_Particle_DP(): No 'DM_cross_section_electron' setting in configuration file.";
		if(!std::isfinite(cfg.sigma_electron_cm2) || cfg.sigma_electron_cm2 < 0.0)
			return "Error in Configuration::Construct_DM_Particle(): DM cross sections must be finite and non-negative.";
		// the proton cross section follows from the electron one (src/Dark_Photon.cpp:130-133, 157-161)
		const double mu_p = cfg.DM_mass_gev * DMS_MPROTON_GEV / (cfg.DM_mass_gev + DMS_MPROTON_GEV);
		const double mu_e = cfg.DM_mass_gev * DMS_MELECTRON_GEV / (cfg.DM_mass_gev + DMS_MELECTRON_GEV);
		cfg.sigma_nucleon_cm2 = cfg.sigma_electron_cm2 * (mu_p / mu_e) * (mu_p / mu_e);
		return Load_Halo(k, cfg);
	}
	cfg.interaction = DMS_INTERACTION_SI;
	k.Bool("DM_isospin_conserved", cfg.DM_isospin_conserved);
	if(!cfg.DM_isospin_conserved)
	{
		const ConfigValue* c = k.Get("DM_relative_couplings");
		if(!c || c->kind != ConfigValue::List || c->items.size() != 2 || c->items[0].kind != ConfigValue::Number || c->items[1].kind != ConfigValue::Number ||
		   c->items[0].number == 0.0)
			return "Error: 'DM_relative_couplings' must be a list (f_p, f_n) with f_p != 0.";
		cfg.fn_over_fp = c->items[1].number / c->items[0].number;
	}
	if(!k.Number("DM_cross_section_nucleon", cfg.sigma_nucleon_cm2))
		return "No 'DM_cross_section_nucleon' setting in configuration file.";
	if(!k.Number("DM_cross_section_electron", cfg.sigma_electron_cm2))
		cfg.sigma_electron_cm2 = 0.0;
	if(!std::isfinite(cfg.sigma_nucleon_cm2) || cfg.sigma_nucleon_cm2 < 0.0 || !std::isfinite(cfg.sigma_electron_cm2) || cfg.sigma_electron_cm2 < 0.0)
		return "Error in Configuration::Construct_DM_Particle(): DM cross sections must be finite and non-negative.";
	k.Str("DM_form_factor", cfg.DM_form_factor);
	if(cfg.DM_form_factor != "Contact")
		return "Error: DM_form_factor " + cfg.DM_form_factor + " is not provided by this engine for SI (Contact is).";
	return Load_Halo(k, cfg);
}

}	// namespace dms
