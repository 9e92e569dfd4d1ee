// Run driver of the engine: the Generate_Data loop of the reference (src/Data_Generation.cpp:488-972)
// over the C ABI, and the reference's output files and summaries
// (src/Data_Generation.cpp:186-348, 1212-1499).
//
// The MPI rounds of the reference become launches of the persistent kernel over contiguous
// trajectory-id ranges.  Capture mode keeps the reference's attempt rule: a round never holds
// more trajectories than captures still missing (src/Data_Generation.cpp:716), so the captured
// count cannot overshoot.  Parameter-point mode sizes rounds in multiples of the reference's
// sigma-dependent sync interval (src/Data_Generation.cpp:59-74) from the capture fraction seen
// so far and stops after the round that reaches the sample size; the excess is reported as
// capture_target_overshoot, as the reference reports the excess of its last MPI round.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <dirent.h>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "../../include/dms.h"
#include "../../include/dms_constants.h"
#include "../../include/dms_driver.h"

namespace
{
constexpr double NUMERICAL_FAILURE_WARNING_FRACTION = 1.0e-4;
constexpr double NUMERICAL_FAILURE_ABORT_FRACTION = 1.0e-2;

uint64_t Sync_Interval(double sigma_cm2)
{
	// Normal_Mode_MPI_Sync_Interval, src/Data_Generation.cpp:59-74
	if(!std::isfinite(sigma_cm2) || sigma_cm2 <= 0.0)
		return 128;
	if(sigma_cm2 >= 1.0e-35)
		return 64;
	if(sigma_cm2 >= 1.0e-36)
		return 128;
	if(sigma_cm2 >= 1.0e-37)
		return 1024;
	if(sigma_cm2 >= 1.0e-38)
		return 8192;
	if(sigma_cm2 >= 1.0e-39)
		return 65536;
	return 1048576;
}

struct Binomial
{
	double rate = 0, err = 0, lo = 0, hi = 0;
};

// Estimate_Binomial_Rate, src/Data_Generation.cpp:186-202 (95 % Wilson interval)
Binomial Estimate(uint64_t trials, uint64_t successes)
{
	Binomial b;
	if(trials == 0)
		return b;
	const double N = static_cast<double>(trials);
	b.rate = static_cast<double>(std::min(successes, trials)) / N;
	b.err = std::sqrt(b.rate * (1.0 - b.rate) / N);
	const double z = 1.96;
	const double den = 1.0 + z * z / N;
	const double center = b.rate + z * z / (2.0 * N);
	const double spread = z * std::sqrt(b.rate * (1.0 - b.rate) / N + z * z / (4.0 * N * N));
	b.lo = std::max(0.0, (center - spread) / den);
	b.hi = std::min(1.0, (center + spread) / den);
	return b;
}

const char* Stop_Key(int r)
{
	switch(r)
	{
		case DMS_STOP_MAX_TRAJECTORIES: return "max_trajectories_reached";
		case DMS_STOP_CAPTURE_TARGET_NOT_REACHED: return "capture_target_not_reached";
		case DMS_STOP_INITIAL_SHIFT_FAILURES: return "initial_shift_failure_fraction_exceeded";
		case DMS_STOP_INVALID_TRAJECTORIES: return "invalid_trajectory_fraction_exceeded";
		default: return "none";
	}
}

const char* Stop_Display(int r)
{
	switch(r)
	{
		case DMS_STOP_MAX_TRAJECTORIES: return "max_trajectories reached";
		case DMS_STOP_CAPTURE_TARGET_NOT_REACHED: return "capture target not reached";
		case DMS_STOP_INITIAL_SHIFT_FAILURES: return "initial shift failure fraction exceeded";
		case DMS_STOP_INVALID_TRAJECTORIES: return "numerical/computational invalid-trajectory fraction exceeded";
		default: return "none";
	}
}

// libphysica::Round semantics used by the summaries: 3 significant digits
double Round3(double d)
{
	if(d == 0.0 || !std::isfinite(d))
		return d;
	const double scale = std::pow(10.0, 2 - std::floor(std::log10(std::fabs(d))));
	return std::round(d * scale) / scale;
}

std::string Time_Display(double s)
{
	std::ostringstream os;
	const long total = static_cast<long>(s);
	const long h = total / 3600, m = (total % 3600) / 60;
	const double sec = s - 3600.0 * h - 60.0 * m;
	if(h > 0)
		os << h << " h ";
	if(h > 0 || m > 0)
		os << m << " min ";
	os << std::fixed << std::setprecision(2) << sec << " s";
	return os.str();
}

bool Ensure_Directory(const std::string& dir)
{
	if(dir.empty())
		return false;
	std::string n = dir;
	while(n.size() > 1 && n.back() == '/') n.pop_back();
	struct stat st;
	if(stat(n.c_str(), &st) == 0)
		return S_ISDIR(st.st_mode);
	const size_t sep = n.find_last_of('/');
	if(sep != std::string::npos && sep > 0 && !Ensure_Directory(n.substr(0, sep)))
		return false;
	return mkdir(n.c_str(), 0755) == 0 || errno == EEXIST;
}

double Snapshot_Bin_Error(double sum, double sum_sq, double count)
{
	// src/Data_Generation.cpp:240-251
	if(count <= 1.0)
		return 0.0;
	const double mean = sum / count;
	double var = sum_sq / count - mean * mean;
	if(var < 0.0)
		var = 0.0;
	return std::sqrt(count * var);
}

uint64_t Valid(const uint64_t* c) { return c[DMS_CNT_CAPTURED] + c[DMS_CNT_COMPLETED_OUTWARD]; }
double Numerical_Failure_Ratio(const uint64_t* c)
{
	return c[DMS_CNT_TRAJECTORIES] > 0 ? 1.0 * c[DMS_CNT_NUMERICAL_FAILURES] / c[DMS_CNT_TRAJECTORIES] : 0.0;
}

// The raw capture-rate lines of bincount.txt and of the snapshot reports, with the legacy
// capture_rate* aliases (src/Data_Generation.cpp:253-278, src/Snapshot_IO.cpp:530-539).
void Write_Raw_Rate_Lines(std::ostream& f, const Binomial& raw)
{
	f << "# capture_rate = " << std::fixed << std::setprecision(8) << raw.rate << "\n";
	f << "# capture_rate_raw = " << std::fixed << std::setprecision(8) << raw.rate << "\n";
	f << "# capture_rate_err = " << std::fixed << std::setprecision(8) << raw.err << "\n";
	f << "# capture_rate_raw_err = " << std::fixed << std::setprecision(8) << raw.err << "\n";
	f << "# capture_rate_CI_95_lower = " << std::fixed << std::setprecision(8) << raw.lo << "\n";
	f << "# capture_rate_CI_95_upper = " << std::fixed << std::setprecision(8) << raw.hi << "\n";
	f << "# capture_rate_raw_CI_95_lower = " << std::fixed << std::setprecision(8) << raw.lo << "\n";
	f << "# capture_rate_raw_CI_95_upper = " << std::fixed << std::setprecision(8) << raw.hi << "\n";
}

void Write_Valid_Rate_Lines(std::ostream& f, const Binomial& valid)
{
	f << "# capture_rate_valid = " << std::fixed << std::setprecision(8) << valid.rate << "\n";
	f << "# capture_rate_valid_err = " << std::fixed << std::setprecision(8) << valid.err << "\n";
	f << "# capture_rate_valid_CI_95_lower = " << std::fixed << std::setprecision(8) << valid.lo << "\n";
	f << "# capture_rate_valid_CI_95_upper = " << std::fixed << std::setprecision(8) << valid.hi << "\n";
}

// The 2000 bin rows (sums and sqrt(N var) errors of captured and not-captured samples),
// src/Data_Generation.cpp:1232-1263 and src/Snapshot_IO.cpp:629-646.
void Write_Bincount_Rows(std::ostream& f, const double* h, double n_cap, double n_nc)
{
	f << "# bin_index  cap_dt[s]  cap_v2dt[km2/s]  cap_err_dt[s]  cap_err_v2dt[km2/s]  not_cap_dt[s]  not_cap_v2dt[km2/s]  not_cap_err_dt[s]  not_cap_err_v2dt[km2/s]\n";
	for(int b = 0; b < DMS_NUM_BINS; b++)
	{
		const double cdt = h[DMS_HIST_CAPTURED_DT * DMS_NUM_BINS + b], cv = h[DMS_HIST_CAPTURED_V2DT * DMS_NUM_BINS + b];
		const double ndt = h[DMS_HIST_NOT_CAPTURED_DT * DMS_NUM_BINS + b], nv = h[DMS_HIST_NOT_CAPTURED_V2DT * DMS_NUM_BINS + b];
		f << b << "\t" << std::scientific << std::setprecision(10) << cdt << "\t" << cv << "\t"
		  << Snapshot_Bin_Error(cdt, h[DMS_HIST_CAPTURED_DT_SQ * DMS_NUM_BINS + b], n_cap) << "\t"
		  << Snapshot_Bin_Error(cv, h[DMS_HIST_CAPTURED_V2DT_SQ * DMS_NUM_BINS + b], n_cap) << "\t" << ndt << "\t" << nv << "\t"
		  << Snapshot_Bin_Error(ndt, h[DMS_HIST_NOT_CAPTURED_DT_SQ * DMS_NUM_BINS + b], n_nc) << "\t"
		  << Snapshot_Bin_Error(nv, h[DMS_HIST_NOT_CAPTURED_V2DT_SQ * DMS_NUM_BINS + b], n_nc) << "\n";
	}
}

// Writes a text file through a temporary name and a rename, so a reader never sees a half
// written report (WriteTextFileAtomically, src/Snapshot_IO.cpp:78-101).
template <class Body>
bool Write_Atomically(const std::string& path, Body body)
{
	const std::string tmp = path + ".tmp." + std::to_string(getpid());
	std::ofstream f(tmp, std::ios::out | std::ios::trunc);
	if(!f.is_open())
		return false;
	body(f);
	f.close();
	if(!f.good() || std::rename(tmp.c_str(), path.c_str()) != 0)
	{
		std::remove(tmp.c_str());
		return false;
	}
	return true;
}

bool Event_Order(const dms_evaporation_event& a, const dms_evaporation_event& b)
{
	if(a.lifetime_unbinding != b.lifetime_unbinding)
		return a.lifetime_unbinding < b.lifetime_unbinding;
	return a.trajectory_id < b.trajectory_id;
}

// Wall-clock progress reports of one Generate_Data call: the reference's heartbeat thread, its
// per-rank checkpoints and rank 0's merge (src/Snapshot_Heartbeat.cpp:236-354,
// src/Snapshot_IO.cpp:369-650) collapse into one writer on the thread that drives the launches,
// called between launches and from the engine's progress hook while a launch is in flight.
// It reads the device accumulators with dms_peek_results, so nothing is recorded per RK step.
// Differences, by design: the trajectories in flight (one per lane, tens of thousands) are
// counted in the rank table but their partial bincounts are not folded into the report (the
// reference folds the one current trajectory of each rank, src/Snapshot_IO.cpp:424-455), and
// an evaporation event is assigned to the first report whose read finds it published.
class Snapshot_Writer
{
  public:
	Snapshot_Writer(dms_ctx* ctx, int point, const dms_generate_opts& g, std::chrono::steady_clock::time_point t0)
	: ctx_(ctx), point_(point), root_(g.snapshot_dir), interval_(g.snapshot_interval_s), mass_(g.snapshot_mass_gev),
	  sigma_(g.snapshot_sigma_cm2), t0_(t0), tolerance_(std::max(1.0, 0.1 * g.snapshot_interval_s)),
	  hist_(DMS_NUM_HISTS * DMS_NUM_BINS)
	{
		if(!root_.empty() && root_.back() != '/')
			root_ += "/";
		run_id_ = static_cast<uint64_t>(
			std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::system_clock::now().time_since_epoch()).count());
		ok_ = Ensure_Directory(root_) && Clear_Previous();
		if(!ok_)
			std::cerr << "Warning in Generate_Data(): failed to initialize snapshot directory; snapshots disabled for this run." << std::endl;
	}

	bool ok() const { return ok_; }
	void Launch_Begins() { launch_active_ = true; }
	void Launch_Ends(uint64_t count)
	{
		launch_active_ = false;
		dispatched_before_ += count;
	}

	// Writes every report whose time has come (a missed-deadline marker for one whose time
	// passed by more than the tolerance before it could be written).
	void Tick()
	{
		if(!ok_)
			return;
		for(double el = Elapsed(); next_ * interval_ <= el; el = Elapsed())
		{
			const double target = next_ * interval_;
			if(el > target + tolerance_ || !Write_Report(next_, launch_active_ ? "running" : "idle_or_waiting", target))
				Write_Missed(next_, Elapsed());
			next_++;
		}
	}

	// The reports that fall due between the last one and the end of the run, written from the
	// final state (FinalizeAfterAllRanksDone, src/Snapshot_Heartbeat.cpp:112-170).
	void Finish(double final_elapsed)
	{
		if(!ok_)
			return;
		const double last = std::floor(final_elapsed / interval_);
		for(; next_ <= last; next_++)
			if(!Write_Report(next_, "done", -1.0))
				std::cerr << "Warning in Generate_Data(): failed to write snapshot " << Label(next_) << "s." << std::endl;
	}

  private:
	long long Label(long long index) const { return index * static_cast<long long>(interval_); }
	std::string Path(long long index, const char* suffix) const { return root_ + "snapshot_" + std::to_string(Label(index)) + "s" + suffix; }
	double Elapsed() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count(); }

	bool Clear_Previous()
	{
		// only this writer's own files: the reference clears the whole snapshot directory
		DIR* d = opendir(root_.c_str());
		if(!d)
			return false;
		std::vector<std::string> names;
		while(dirent* e = readdir(d))
			if(std::strncmp(e->d_name, "snapshot_", 9) == 0)
				names.push_back(e->d_name);
		closedir(d);
		bool ok = true;
		for(const auto& n : names)
			ok = (std::remove((root_ + n).c_str()) == 0) && ok;
		return ok;
	}

	// snapshot_status / run id lines common to both files of a report (one rank: always merged)
	void Write_Status(std::ostream& f) const
	{
		f << "# snapshot_status = merged\n";
		f << "# snapshot_run_id = " << run_id_ << "\n";
	}

	// deadline_s < 0: the final report, written whatever the time
	bool Write_Report(long long index, const char* state, double deadline_s)
	{
		dms_point_results r;
		std::memset(&r, 0, sizeof r);
		if(dms_peek_results(ctx_, point_, &r) != DMS_OK)
			return false;
		events_.resize(std::max<uint64_t>(r.events_count, 1) + 1024);
		std::memset(&r, 0, sizeof r);
		r.histograms = hist_.data();
		r.events = events_.data();
		r.events_capacity = events_.size();
		dms_progress pr;
		if(dms_peek_results(ctx_, point_, &r) != DMS_OK || dms_peek_progress(ctx_, &pr) != DMS_OK)
			return false;
		const double observed = Elapsed();
		if(deadline_s >= 0.0 && observed > deadline_s + tolerance_)
			return false;
		const uint64_t* c = r.counters;
		const uint64_t published = std::max<uint64_t>(r.events_count, published_);
		std::vector<dms_evaporation_event> fresh(events_.begin() + published_, events_.begin() + published);
		std::sort(fresh.begin(), fresh.end(), Event_Order);
		const bool done = deadline_s < 0.0;
		const uint64_t dispatched = dispatched_before_ + (launch_active_ && pr.running ? pr.dispatched : 0);
		const uint64_t completed = c[DMS_CNT_TRAJECTORIES];
		const uint64_t in_flight = (!done && dispatched > completed) ? dispatched - completed : 0;

		// WriteSnapshotEvaporationTimeFile, src/Snapshot_IO.cpp:545-576
		const bool events_ok = Write_Atomically(Path(index, "_evaporation_times.txt"), [&](std::ofstream& f) {
			Write_Status(f);
			f << "# snapshot_target_wall_time_s = " << Label(index) << "\n";
			f << "# snapshot_interval_s = " << std::fixed << std::setprecision(3) << interval_ << "\n";
			f << "# ready_ranks = 0\n";
			f << "# missing_ranks = \n";
			f << "# completed_evaporation_events_assigned_to_snapshot = 1\n";
			f << "# event_assignment = first published checkpoint after completion\n";
			f << "# DaMaSCUS-SUN snapshot evaporation times\n";
			f << "# format_version = 3\n";
			f << "# DIAGNOSTIC_ONLY = 1\n";
			f << "# NOT_FOR_FINAL_SURVIVAL_ANALYSIS = 1\n";
			f << "# completion_time_selected = 1\n";
			f << "# DM_mass_GeV = " << std::scientific << std::setprecision(6) << mass_ << "\n";
			f << "# DM_sigma_cm2 = " << std::scientific << std::setprecision(6) << sigma_ << "\n";
			f << "# sorted_by = lifetime_unbinding_sec rank trajectory_id\n";
			f << "# rank trajectory_id lifetime_unbinding_sec\n";
			for(const auto& e : fresh)
				if(std::isfinite(e.lifetime_unbinding) && e.lifetime_unbinding >= 0.0)
					f << 0 << "\t" << e.trajectory_id << "\t" << std::scientific << std::setprecision(10) << e.lifetime_unbinding << "\n";
		});
		if(!events_ok)
			return false;
		published_ = published;

		// WriteSnapshotReportFile + WriteReportHeader, src/Snapshot_IO.cpp:508-543, 578-650
		return Write_Atomically(Path(index, ".txt"), [&](std::ofstream& f) {
			const uint64_t valid = Valid(c);
			Write_Status(f);
			f << "# Cumulative snapshot report\n";
			f << "# ready_ranks = 0\n";
			f << "# missing_ranks = \n";
			f << "# snapshot_target_wall_time_s = " << Label(index) << "\n";
			f << "# snapshot_interval_s = " << std::fixed << std::setprecision(3) << interval_ << "\n";
			f << "# DM_mass_GeV = " << std::scientific << std::setprecision(6) << mass_ << "\n";
			f << "# DM_sigma_cm2 = " << std::scientific << std::setprecision(6) << sigma_ << "\n";
			f << "# total_trajectories = " << completed << "\n";
			f << "# captured_particles = " << c[DMS_CNT_CAPTURED] << "\n";
			f << "# valid_trajectories = " << valid << "\n";
			f << "# numerical_failures = " << c[DMS_CNT_NUMERICAL_FAILURES] << "\n";
			f << "# unresolved_not_captured_trajectories = " << (completed > valid ? completed - valid : 0) << "\n";
			Write_Raw_Rate_Lines(f, Estimate(completed, c[DMS_CNT_CAPTURED]));
			Write_Valid_Rate_Lines(f, Estimate(valid, c[DMS_CNT_CAPTURED]));
			f << "#\n";
			f << "# [GPU rank status]\n";
			f << "# rank  state  dispatched_trajectories  in_flight_trajectories  completed_trajectories  completed_scatterings  observed_at_wall_s\n";
			f << "# 0\t" << state << "\t" << dispatched << "\t" << in_flight << "\t" << completed << "\t" << c[DMS_CNT_TOTAL_SCATTERINGS]
			  << "\t" << std::scientific << std::setprecision(10) << observed << "\n";
			f << "#\n";
			f << "# [Bincount histogram]\n";
			Write_Bincount_Rows(f, hist_.data(), static_cast<double>(c[DMS_CNT_CAPTURED]), static_cast<double>(c[DMS_CNT_COMPLETED_OUTWARD]));
		});
	}

	// WriteMissedSnapshotMarker, src/Snapshot_IO.cpp:925-947
	void Write_Missed(long long index, double actual_s)
	{
		Write_Atomically(Path(index, ".txt"), [&](std::ofstream& f) {
			f << "# snapshot_status = missed_writer_delay\n";
			f << "# snapshot_run_id = " << run_id_ << "\n";
			f << "# snapshot_target_wall_time_s = " << Label(index) << "\n";
			f << "# snapshot_interval_s = " << std::fixed << std::setprecision(3) << interval_ << "\n";
			f << "# actual_write_wall_time_s = " << std::fixed << std::setprecision(3) << actual_s << "\n";
			f << "# note = heartbeat woke too late; no state rewind is available\n";
		});
	}

	dms_ctx* ctx_;
	int point_;
	std::string root_;
	double interval_, mass_, sigma_;
	std::chrono::steady_clock::time_point t0_;
	double tolerance_;
	uint64_t run_id_ = 0;
	bool ok_ = false;
	bool launch_active_ = false;
	long long next_ = 1;
	uint64_t dispatched_before_ = 0;
	uint64_t published_ = 0;
	std::vector<double> hist_;
	std::vector<dms_evaporation_event> events_;
};


// Removes the progress hook when the generate call returns, on every path.
struct Hook_Guard
{
	dms_ctx* ctx;
	~Hook_Guard()
	{
		if(ctx)
			dms_set_progress_callback(ctx, nullptr, nullptr, 0.0);
	}
};

// print_progress_update, src/Data_Generation.cpp:661-694: one line when the captured fraction of
// the requested sample passes a milestone, with a progress bar, the elapsed time and the capture
// rate.  The bar is this library's own drawing (libphysica's is not part of the reference).
class Progress_Printer
{
  public:
	Progress_Printer(bool on, uint32_t requested, std::chrono::steady_clock::time_point t0) : on_(on), requested_(requested), t0_(t0) {}
	void Update(uint64_t captured, bool force)
	{
		if(!on_)
			return;
		static const double milestones[] = {0.0, 0.01, 0.05, 0.10, 0.20, 0.40, 0.60, 0.80, 1.0};
		const double progress = std::min(1.0, static_cast<double>(captured) / std::max<double>(1.0, requested_));
		bool print = force;
		while(next_ < sizeof milestones / sizeof milestones[0] && progress + 1.0e-12 >= milestones[next_])
		{
			print = true;
			next_++;
		}
		if(!print || (force && printed_ && captured == last_))
			return;
		const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
		const int width = 44, filled = static_cast<int>(progress * width + 0.5);
		std::cout << "[" << std::string(filled, '=') << std::string(width - filled, ' ') << "] " << std::setw(3)
		          << static_cast<int>(100.0 * progress + 0.5) << " % (" << Time_Display(el) << ")"
		          << " captured_particles=" << captured << "/" << requested_
		          << " captured_particle_rate[1/s]=" << Round3(el > 0.0 ? captured / el : 0.0) << std::endl;
		printed_ = true;
		last_ = captured;
	}

  private:
	bool on_;
	uint32_t requested_;
	std::chrono::steady_clock::time_point t0_;
	size_t next_ = 0;
	bool printed_ = false;
	uint64_t last_ = 0;
};

// What the driver does while a launch is in flight: snapshot reports that fall due, and the
// progress lines of captures reached (read with dms_peek_results beside the kernel).
struct Launch_Hook
{
	Snapshot_Writer* snapshots;
	Progress_Printer* progress;
	int point;
};

int Launch_Hook_Call(dms_ctx* ctx, void* user)
{
	const Launch_Hook& h = *static_cast<Launch_Hook*>(user);
	if(h.snapshots)
		h.snapshots->Tick();
	if(h.progress)
	{
		dms_point_results r;
		std::memset(&r, 0, sizeof r);
		if(dms_peek_results(ctx, h.point, &r) == DMS_OK)
			h.progress->Update(r.counters[DMS_CNT_CAPTURED], false);
	}
	return 0;
}

bool Snapshot_Interval_Valid(double s)
{
	// IsValidSnapshotIntervalSeconds, src/Snapshot_IO.cpp:652-658
	return std::isfinite(s) && s >= 1.0 && s <= 2147483647.0 && std::floor(s) == s;
}
}	// namespace

extern "C" {

void dms_default_generate_opts(dms_generate_opts* o)
{
	if(!o)
		return;
	std::memset(o, 0, sizeof *o);
	o->sample_size = 1;
	o->max_scatterings = 100000000000000ULL;
	o->boundary_radius_rsun = 2.0;
	o->round_capacity = 1u << 20;
}

int dms_generate_data(dms_ctx* ctx, int point_id, const dms_generate_opts* g, dms_generate_summary* out)
{
	if(!ctx || !g || !out)
		return DMS_ERR_INVALID_ARGUMENT;
	if(g->sample_size == 0)
		return DMS_ERR_INVALID_ARGUMENT;
	std::memset(out, 0, sizeof *out);
	int rc = dms_reset_results(ctx, point_id);
	if(rc != DMS_OK)
		return rc;
	dms_run_opts opts;
	dms_default_run_opts(&opts);
	opts.seed = g->seed;
	opts.capture_mode = g->capture_mode ? 1 : 0;
	opts.max_scatterings = g->max_scatterings;
	opts.boundary_radius_rsun = g->boundary_radius_rsun;
	opts.time_limit_s = g->time_limit_s;
	opts.max_trajectory_wall_time_s = g->max_trajectory_wall_time_s;
	if(g->max_free_steps != 0)
		opts.max_free_steps = g->max_free_steps;
	opts.threads_per_block = g->threads_per_block;
	opts.blocks_per_sm = g->blocks_per_sm;
	const uint64_t interval = g->capture_mode ? 32 : Sync_Interval(g->sigma_p_cm2);
	out->sync_interval = g->capture_mode ? 0 : interval;
	const uint64_t budget = g->max_trajectories == 0 ? UINT64_MAX : g->max_trajectories;
	const uint64_t round_cap = std::max<uint64_t>(interval, g->round_capacity ? g->round_capacity : (1u << 20));
	dms_point_results res;
	std::memset(&res, 0, sizeof res);
	uint64_t next_id = 0;
	int stop = DMS_STOP_NONE;
	bool warned = false;
	const auto t0 = std::chrono::steady_clock::now();
	std::unique_ptr<Snapshot_Writer> snapshots;
	Hook_Guard guard{nullptr};
	if(g->snapshot_dir && !g->capture_mode)
	{
		if(!Snapshot_Interval_Valid(g->snapshot_interval_s))
			return DMS_ERR_INVALID_ARGUMENT;
		snapshots.reset(new Snapshot_Writer(ctx, point_id, *g, t0));
		if(!snapshots->ok())
			snapshots.reset();
	}
	Progress_Printer progress(g->print_progress != 0, g->sample_size, t0);
	progress.Update(0, true);
	Launch_Hook hook{snapshots.get(), g->print_progress ? &progress : nullptr, point_id};
	if(hook.snapshots || hook.progress)
	{
		const double interval = hook.snapshots ? std::min(0.1, 0.1 * g->snapshot_interval_s) : 0.25;
		rc = dms_set_progress_callback(ctx, Launch_Hook_Call, &hook, interval);
		if(rc != DMS_OK)
			return rc;
		guard.ctx = ctx;
	}
	for(;;)
	{
		if(snapshots)
			snapshots->Tick();
		rc = dms_get_results(ctx, point_id, &res);
		if(rc != DMS_OK)
			return rc;
		progress.Update(res.counters[DMS_CNT_CAPTURED], false);
		const uint64_t* c = res.counters;
		const uint64_t captured = c[DMS_CNT_CAPTURED];
		const uint64_t done = c[DMS_CNT_TRAJECTORIES];
		if(done > 0)
		{
			// run-level fuses, src/Data_Generation.cpp:893-938
			const double shift_frac = 1.0 * c[DMS_CNT_INITIAL_SHIFT_FAILURES] / done;
			if(shift_frac > NUMERICAL_FAILURE_ABORT_FRACTION)
			{
				std::cerr << "Error in Generate_Data(): initial Kepler shift failure fraction " << shift_frac << " exceeds abort threshold "
				          << NUMERICAL_FAILURE_ABORT_FRACTION << ". Stopping this run to avoid biased capture statistics." << std::endl;
				stop = DMS_STOP_INITIAL_SHIFT_FAILURES;
				break;
			}
			if(!warned && shift_frac > NUMERICAL_FAILURE_WARNING_FRACTION)
			{
				std::cerr << "Warning in Generate_Data(): initial Kepler shift failure fraction " << shift_frac << " exceeds warning threshold "
				          << NUMERICAL_FAILURE_WARNING_FRACTION << "." << std::endl;
				warned = true;
			}
			const double invalid = 1.0 * (c[DMS_CNT_NUMERICAL_FAILURES] + c[DMS_CNT_COMPUTATIONAL_TRUNCATIONS]) / done;
			if(budget == UINT64_MAX && invalid > NUMERICAL_FAILURE_ABORT_FRACTION)
			{
				std::cerr << "Error in Generate_Data(): invalid trajectory fraction " << invalid << " exceeds abort threshold "
				          << NUMERICAL_FAILURE_ABORT_FRACTION << " with an unlimited trajectory budget. Stopping to avoid a non-progressing run." << std::endl;
				stop = DMS_STOP_INVALID_TRAJECTORIES;
				break;
			}
		}
		if(captured >= g->sample_size)
			break;
		if(next_id >= budget)
		{
			stop = DMS_STOP_MAX_TRAJECTORIES;
			break;
		}
		const uint64_t remaining = g->sample_size - captured;
		uint64_t round;
		if(g->capture_mode)
			round = std::min<uint64_t>(remaining, round_cap);
		else
		{
			const double p = (done > 0 && captured > 0) ? static_cast<double>(captured) / done : 0.0;
			const double need = (p > 0.0) ? remaining / p : static_cast<double>(interval) * 64.0;
			uint64_t r = static_cast<uint64_t>(std::ceil(need / interval)) * interval;
			r = std::max<uint64_t>(r, interval);
			round = std::min<uint64_t>(r, round_cap);
		}
		round = std::min<uint64_t>(round, budget - next_id);
		dms_work_range range;
		range.point_id = point_id;
		range.reserved = 0;
		range.first_trajectory = next_id;
		range.count = round;
		if(snapshots)
			snapshots->Launch_Begins();
		rc = dms_run(ctx, &opts, &range, 1);
		if(snapshots)
			snapshots->Launch_Ends(round);
		if(rc != DMS_OK)
			return rc;
		next_id += round;
		out->rounds++;
		out->final_round_trajectories = round;
	}
	out->computing_time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	{
		dms_point_results last;
		std::memset(&last, 0, sizeof last);
		if(dms_get_results(ctx, point_id, &last) == DMS_OK)
			progress.Update(last.counters[DMS_CNT_CAPTURED], true);
	}
	if(snapshots)
	{
		dms_set_progress_callback(ctx, nullptr, nullptr, 0.0);
		snapshots->Finish(out->computing_time_s);
	}
	rc = dms_get_results(ctx, point_id, &res);
	if(rc != DMS_OK)
		return rc;
	std::memcpy(out->counters, res.counters, sizeof out->counters);
	const uint64_t captured = out->counters[DMS_CNT_CAPTURED];
	out->capture_target_overshoot = captured > g->sample_size ? captured - g->sample_size : 0;
	if(captured < g->sample_size && stop == DMS_STOP_NONE)
		stop = DMS_STOP_CAPTURE_TARGET_NOT_REACHED;
	out->early_stop_reason = stop;
	out->next_trajectory = next_id;
	return DMS_OK;
}

int dms_write_outputs(dms_ctx* ctx, int point_id, const dms_generate_summary* s, double mass_gev, double sigma_cm2, const char* output_dir)
{
	if(!ctx || !s || !output_dir)
		return DMS_ERR_INVALID_ARGUMENT;
	std::string dir = output_dir;
	if(!Ensure_Directory(dir))
	{
		std::cerr << "Warning in Write_Output_Files(): failed to create output directory " << dir << std::endl;
		return DMS_ERR_IO;
	}
	std::vector<double> hist(DMS_NUM_HISTS * DMS_NUM_BINS);
	dms_point_results res;
	std::memset(&res, 0, sizeof res);
	res.histograms = hist.data();
	int rc = dms_get_results(ctx, point_id, &res);
	if(rc != DMS_OK)
		return rc;
	std::vector<dms_evaporation_event> events(res.events_count);
	res.events = events.data();
	res.events_capacity = events.size();
	rc = dms_get_results(ctx, point_id, &res);
	if(rc != DMS_OK)
		return rc;
	const uint64_t* c = s->counters;
	const uint64_t N = c[DMS_CNT_TRAJECTORIES];
	const uint64_t unresolved = N > Valid(c) ? N - Valid(c) : 0;
	auto join = [&](const char* name) { return (dir.back() == '/') ? dir + name : dir + "/" + name; };
	{
		// Write_Report_Header + the bincount.txt body, src/Data_Generation.cpp:253-278, 1232-1263
		std::ofstream f(join("bincount.txt"));
		const Binomial raw = Estimate(N, c[DMS_CNT_CAPTURED]);
		f << "# DM_mass_GeV = " << std::scientific << std::setprecision(6) << mass_gev << "\n";
		f << "# DM_sigma_cm2 = " << std::scientific << std::setprecision(6) << sigma_cm2 << "\n";
		f << "# total_trajectories = " << N << "\n";
		f << "# captured_particles = " << c[DMS_CNT_CAPTURED] << "\n";
		Write_Raw_Rate_Lines(f, raw);
		if(s->early_stop_reason != DMS_STOP_NONE)
			f << "# EARLY_STOP: " << Stop_Key(s->early_stop_reason) << "\n";
		f << "# valid_trajectories = " << Valid(c) << "\n";
		f << "# completed_outward_escapes = " << c[DMS_CNT_COMPLETED_OUTWARD] << "\n";
		f << "# unresolved_not_captured_trajectories = " << unresolved << "\n";
		f << "# numerical_failures = " << c[DMS_CNT_NUMERICAL_FAILURES] << "\n";
		f << "# computational_truncations = " << c[DMS_CNT_COMPUTATIONAL_TRUNCATIONS] << "\n";
		f << "# initial_shift_failures = " << c[DMS_CNT_INITIAL_SHIFT_FAILURES] << "\n";
		f << "# final_reflection_shift_failures = " << c[DMS_CNT_FINAL_REFLECTION_SHIFT_FAILURES] << "\n";
		f << "# normal_mode_mpi_sync_interval = " << s->sync_interval << "\n";
		f << "# mpi_sync_rounds = " << s->rounds << "\n";
		f << "# final_mpi_round_trajectories = " << s->final_round_trajectories << "\n";
		f << "# mpi_tail_trajectories = " << 0 << "\n";
		f << "# capture_target_overshoot = " << s->capture_target_overshoot << "\n";
		f << "# total_scatterings = " << c[DMS_CNT_TOTAL_SCATTERINGS] << "\n";
		const double avg = N > 0 ? static_cast<double>(c[DMS_CNT_TOTAL_SCATTERINGS]) / N : 0.0;
		f << "# average_scatterings = " << std::setprecision(12) << avg << "\n";
		f << "# simulation_time_seconds = " << std::setprecision(12) << s->computing_time_s << "\n";
		Write_Valid_Rate_Lines(f, Estimate(Valid(c), c[DMS_CNT_CAPTURED]));
		f << "# numerical_failure_rate = " << std::fixed << std::setprecision(8) << Numerical_Failure_Ratio(c) << "\n";
		f << "# not_captured_bincount_samples = " << c[DMS_CNT_COMPLETED_OUTWARD] << "\n";
		if(unresolved > 0)
			f << "# excluded_incomplete_not_captured = " << unresolved << "\n";
		Write_Bincount_Rows(f, hist.data(), static_cast<double>(c[DMS_CNT_CAPTURED]), static_cast<double>(c[DMS_CNT_COMPLETED_OUTWARD]));
		if(!f.good())
			return DMS_ERR_IO;
	}
	{
		// Write_Final_Evaporation_Time_File, src/Data_Generation.cpp:292-348 (one rank: rank 0)
		std::sort(events.begin(), events.end(), Event_Order);
		const std::string path = join("evaporation_times.txt");
		const std::string tmp = path + ".final.tmp." + std::to_string(getpid());
		std::ofstream f(tmp, std::ios::out | std::ios::trunc);
		f << "# DaMaSCUS-SUN evaporation times\n";
		f << "# format_version = 3\n";
		f << "# DM_mass_GeV = " << std::scientific << std::setprecision(6) << mass_gev << "\n";
		f << "# DM_sigma_cm2 = " << std::scientific << std::setprecision(6) << sigma_cm2 << "\n";
		f << "# sorted_by = lifetime_unbinding_sec rank trajectory_id\n";
		f << "# rank trajectory_id lifetime_unbinding_sec\n";
		for(const auto& e : events)
			if(std::isfinite(e.lifetime_unbinding) && e.lifetime_unbinding >= 0.0)
				f << 0 << "\t" << e.trajectory_id << "\t" << std::scientific << std::setprecision(10) << e.lifetime_unbinding << "\n";
		f.close();
		if(!f.good() || std::rename(tmp.c_str(), path.c_str()) != 0)
		{
			std::remove(tmp.c_str());
			std::cerr << "Warning in Write_Output_Files(): failed to write evaporation_times.txt" << std::endl;
			return DMS_ERR_IO;
		}
	}
	return DMS_OK;
}

int dms_print_summary(dms_ctx* ctx, int point_id, const dms_generate_summary* s, int capture_mode)
{
	if(!s)
		return DMS_ERR_INVALID_ARGUMENT;
	const uint64_t* c = s->counters;
	const uint64_t N = c[DMS_CNT_TRAJECTORIES];
	const Binomial raw = Estimate(N, c[DMS_CNT_CAPTURED]);
	const Binomial valid = Estimate(Valid(c), c[DMS_CNT_CAPTURED]);
	const char* sep = "\n----------------------------------------\n";
	const double t = s->computing_time_s;
	if(capture_mode)
	{
		// Print_Capture_Mode_Summary, src/Data_Generation.cpp:1366-1404
		std::cout << sep << "CAPTURE MODE summary" << std::endl
		          << std::endl
		          << "Termination condition:\t\tpost-scatter E < 0" << std::endl
		          << "File output:\t\t\tdisabled" << std::endl
		          << "Simulated trajectories:\t\t" << N << std::endl
		          << "Capture-classified trajectories:\t" << Valid(c) << std::endl
		          << "Unresolved non-captures:\t\t" << (N - Valid(c)) << std::endl
		          << "Captured count:\t\t\t" << c[DMS_CNT_CAPTURED] << std::endl
		          << "Capture rate raw:\t\t" << std::fixed << std::setprecision(8) << raw.rate << std::endl
		          << "Capture rate valid:\t\t" << std::fixed << std::setprecision(8) << valid.rate << std::endl
		          << "Capture rate raw 95% CI:\t[" << raw.lo << ", " << raw.hi << "]" << std::endl
		          << "Capture rate valid 95% CI:\t[" << valid.lo << ", " << valid.hi << "]" << std::endl
		          << "Numerical failure count:\t" << c[DMS_CNT_NUMERICAL_FAILURES] << std::endl
		          << "Computational truncations:\t" << c[DMS_CNT_COMPUTATIONAL_TRUNCATIONS] << std::endl
		          << "Initial shift failures:\t\t" << c[DMS_CNT_INITIAL_SHIFT_FAILURES] << std::endl
		          << "Final reflection shift failures:\t" << c[DMS_CNT_FINAL_REFLECTION_SHIFT_FAILURES] << std::endl
		          << "Numerical failure rate:\t\t" << std::fixed << std::setprecision(8) << Numerical_Failure_Ratio(c) << std::endl;
		if(s->early_stop_reason != DMS_STOP_NONE)
			std::cout << "*** EARLY STOP: " << Stop_Display(s->early_stop_reason) << " ***" << std::endl;
		if(Numerical_Failure_Ratio(c) > NUMERICAL_FAILURE_WARNING_FRACTION)
			std::cout << "*** WARNING: numerical failure rate exceeded " << NUMERICAL_FAILURE_WARNING_FRACTION << " ***" << std::endl;
		std::cout << "Captured particle rate [1/s]:\t" << Round3(t > 0 ? c[DMS_CNT_CAPTURED] / t : 0.0) << std::endl
		          << "Total # of scatterings:\t" << c[DMS_CNT_TOTAL_SCATTERINGS] << std::endl
		          << "Simulation time [s]:\t\t" << std::fixed << std::setprecision(6) << t << std::endl
		          << "Simulation time:\t\t" << Time_Display(t) << std::endl
		          << sep << std::endl;
		return DMS_OK;
	}
	// Print_Summary, src/Data_Generation.cpp:1406-1497
	std::vector<dms_evaporation_event> events;
	if(ctx)
	{
		dms_point_results res;
		std::memset(&res, 0, sizeof res);
		if(dms_get_results(ctx, point_id, &res) == DMS_OK && res.events_count > 0)
		{
			events.resize(res.events_count);
			res.events = events.data();
			res.events_capacity = events.size();
			dms_get_results(ctx, point_id, &res);
		}
	}
	const double avg = N > 0 ? static_cast<double>(c[DMS_CNT_TOTAL_SCATTERINGS]) / N : 0.0;
	auto pct = [&](uint64_t k, uint64_t d) { return d > 0 ? Round3(100.0 * k / d) : 0.0; };
	std::cout << sep << "Simulation data summary" << std::endl
	          << std::endl
	          << "Results:" << std::endl
	          << "Simulated trajectories:\t\t" << N << std::endl
	          << "Capture-classified trajectories:\t" << Valid(c) << std::endl
	          << "Unresolved non-captures:\t\t" << (N - Valid(c)) << std::endl
	          << "Average # of scatterings:\t" << Round3(avg) << std::endl
	          << "Free particles raw [%]:\t\t" << pct(c[DMS_CNT_FREE], N) << std::endl
	          << "Reflected particles raw [%]:\t" << pct(c[DMS_CNT_REFLECTED], N) << std::endl
	          << "Captured particles raw [%]:\t" << pct(c[DMS_CNT_CAPTURED], N) << std::endl
	          << "Free particles valid [%]:\t" << pct(c[DMS_CNT_FREE], Valid(c)) << std::endl
	          << "Reflected particles valid [%]:\t" << pct(c[DMS_CNT_REFLECTED], Valid(c)) << std::endl
	          << "Captured particles valid [%]:\t" << pct(c[DMS_CNT_CAPTURED], Valid(c)) << std::endl
	          << "Captured count:\t\t\t" << c[DMS_CNT_CAPTURED] << std::endl
	          << "Normal-mode MPI sync interval:\t" << s->sync_interval << std::endl
	          << "MPI sync rounds:\t\t" << s->rounds << std::endl
	          << "Final MPI round trajectories:\t" << s->final_round_trajectories << std::endl
	          << "MPI tail trajectories:\t\t" << 0 << std::endl
	          << "Capture target overshoot:\t" << s->capture_target_overshoot << std::endl
	          << "Total # of scatterings:\t" << c[DMS_CNT_TOTAL_SCATTERINGS] << std::endl
	          << "Numerical failure count:\t" << c[DMS_CNT_NUMERICAL_FAILURES] << std::endl
	          << "Computational truncations:\t" << c[DMS_CNT_COMPUTATIONAL_TRUNCATIONS] << std::endl
	          << "Initial shift failures:\t\t" << c[DMS_CNT_INITIAL_SHIFT_FAILURES] << std::endl
	          << "Final reflection shift failures:\t" << c[DMS_CNT_FINAL_REFLECTION_SHIFT_FAILURES] << std::endl
	          << "Numerical failure rate:\t\t" << std::fixed << std::setprecision(6) << Numerical_Failure_Ratio(c) << std::endl
	          << "Complete evaporation count:\t" << c[DMS_CNT_COMPLETE_EVAPORATION] << std::endl
	          << "Censored captured count:\t" << c[DMS_CNT_CENSORED_CAPTURED] << std::endl
	          << "Invalid survival count:\t\t" << c[DMS_CNT_INVALID_SURVIVAL] << std::endl;
	std::cout << "Capture rate raw error (1\xcf\x83):\t" << std::fixed << std::setprecision(6) << raw.err << std::endl
	          << "Capture rate raw 95% CI:\t[" << raw.lo << ", " << raw.hi << "]" << std::endl
	          << "Capture rate valid error (1\xcf\x83):\t" << valid.err << std::endl
	          << "Capture rate valid 95% CI:\t[" << valid.lo << ", " << valid.hi << "]" << std::endl;
	if(s->early_stop_reason != DMS_STOP_NONE)
		std::cout << "*** EARLY STOP: " << Stop_Display(s->early_stop_reason) << " ***" << std::endl;
	if(Numerical_Failure_Ratio(c) > NUMERICAL_FAILURE_WARNING_FRACTION)
		std::cout << "*** WARNING: numerical failure rate exceeded " << NUMERICAL_FAILURE_WARNING_FRACTION << " ***" << std::endl;
	std::vector<double> lifetimes;
	for(const auto& e : events)
		if(std::isfinite(e.lifetime_unbinding) && e.lifetime_unbinding > 0.0)
			lifetimes.push_back(e.lifetime_unbinding);
	if(!lifetimes.empty())
	{
		std::sort(lifetimes.begin(), lifetimes.end());
		const size_t n = lifetimes.size();
		const double median = (n % 2 == 0) ? 0.5 * (lifetimes[n / 2 - 1] + lifetimes[n / 2]) : lifetimes[n / 2];
		std::cout << "Observed unbinding lifetime median [s]:\t" << std::scientific << std::setprecision(4) << median << " (" << n << " events)" << std::endl;
	}
	else
		std::cout << "Observed unbinding lifetime median:\tN/A (no positive observed unbinding events)" << std::endl;
	std::cout << std::endl
	          << "Trajectory rate [1/s]:\t\t" << Round3(t > 0 ? N / t : 0.0) << std::endl
	          << "Captured particle rate [1/s]:\t" << Round3(t > 0 ? c[DMS_CNT_CAPTURED] / t : 0.0) << std::endl
	          << "Scattering rate [1/s]:\t\t" << Round3(t > 0 ? c[DMS_CNT_TOTAL_SCATTERINGS] / t : 0.0) << std::endl
	          << "Simulation time [s]:\t\t" << std::fixed << std::setprecision(6) << t << std::endl
	          << "Simulation time:\t\t" << Time_Display(t) << std::endl
	          << sep << std::endl;
	return DMS_OK;
}

}	// extern "C"
