"""Ensemble comparison of two engine runs of one parameter point (mixed precision against FP64).

The reference validates ensembles with binomial capture rates and per-bin errors of the
time-weighted radial histogram (Estimate_Binomial_Rate and Snapshot_Bin_Error,
src/Data_Generation.cpp:186-202, 240-251; validation/physics_validation.py:192-309).  The same
estimators give the error of a mixed-precision run against the FP64 run of the same
trajectories:

* capture fraction: relative difference and its size in binomial standard errors;
* radial histogram (captured, time-weighted dt per bin, normalised per trajectory): chi-squared
  over the bins with a nonzero error, its p-value, and the largest per-bin pull;
* evaporation rate (completed unbinding events per trajectory) and mean scatterings per
  trajectory: relative differences.

Inputs are the dictionaries returned by dms_b200.Engine.results()."""
import math

import numpy as np

HIST_CAPTURED_DT = 0
HIST_CAPTURED_DT_SQ = 4


def _chi2_sf(x, k):
    """Survival function of the chi-squared distribution with k degrees of freedom."""
    try:
        from scipy.stats import chi2
        return float(chi2.sf(x, k))
    except ImportError:  # Wilson-Hilferty normal approximation
        if k <= 0:
            return 1.0
        z = ((x / k) ** (1.0 / 3.0) - (1.0 - 2.0 / (9.0 * k))) / math.sqrt(2.0 / (9.0 * k))
        return 0.5 * math.erfc(z / math.sqrt(2.0))


def binned_means(res, slot=HIST_CAPTURED_DT, slot_sq=HIST_CAPTURED_DT_SQ):
    """Per-trajectory mean of one histogram and the variance of that mean, per bin."""
    n = res["counters"]["trajectories"]
    s = np.asarray(res["histograms"][slot], dtype=np.float64)
    s2 = np.asarray(res["histograms"][slot_sq], dtype=np.float64)
    if n == 0:
        return np.zeros_like(s), np.zeros_like(s)
    mean = s / n
    var_sum = np.maximum(s2 - s * s / n, 0.0)   # N * sample variance of one trajectory's bin value
    return mean, var_sum / (n * n)


def compare_runs(ref, other):
    """Error of `other` against `ref` (both Engine.results() dictionaries of the same point)."""
    ca, cb = ref["counters"], other["counters"]
    na, nb = ca["trajectories"], cb["trajectories"]
    fa = ca["captured"] / na if na else 0.0
    fb = cb["captured"] / nb if nb else 0.0
    sigma = math.sqrt(max(fa * (1.0 - fa), 0.0) / na + max(fb * (1.0 - fb), 0.0) / nb) if na and nb else 0.0
    out = {
        "trajectories": [na, nb],
        "capture_fraction": [fa, fb],
        "capture_fraction_rel_error": abs(fb - fa) / fa if fa > 0 else (0.0 if fb == 0 else math.inf),
        "capture_fraction_sigmas": abs(fb - fa) / sigma if sigma > 0 else (0.0 if fa == fb else math.inf),
    }
    ma, va = binned_means(ref)
    mb, vb = binned_means(other)
    var = va + vb
    used = var > 0
    pulls = np.zeros_like(ma)
    pulls[used] = (mb[used] - ma[used]) / np.sqrt(var[used])
    chi2 = float(np.sum(pulls[used] ** 2))
    dof = int(np.count_nonzero(used))
    out["radial_chi2"] = chi2
    out["radial_dof"] = dof
    out["radial_p_value"] = _chi2_sf(chi2, dof) if dof else 1.0
    out["radial_max_pull"] = float(np.max(np.abs(pulls))) if dof else 0.0
    sa, sb = float(np.sum(ma)), float(np.sum(mb))
    out["radial_max_bin_deviation"] = float(np.max(np.abs(mb / sb - ma / sa))) if sa > 0 and sb > 0 else 0.0
    ea = len(ref["events"]) / na if na else 0.0
    eb = len(other["events"]) / nb if nb else 0.0
    out["evaporation_rate"] = [ea, eb]
    out["evaporation_rate_rel_error"] = abs(eb - ea) / ea if ea > 0 else (0.0 if eb == 0 else math.inf)
    sa_ = ca["total_scatterings"] / na if na else 0.0
    sb_ = cb["total_scatterings"] / nb if nb else 0.0
    out["mean_scatterings"] = [sa_, sb_]
    out["mean_scatterings_rel_error"] = abs(sb_ - sa_) / sa_ if sa_ > 0 else 0.0
    return out
