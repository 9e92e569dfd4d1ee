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


def wilson_interval(successes, trials, z=1.959963984540054):
    """95 % Wilson score interval of a binomial rate."""
    if trials <= 0:
        return 0.0, 0.0
    p = successes / trials
    den = 1.0 + z * z / trials
    centre = (p + z * z / (2.0 * trials)) / den
    half = z * math.sqrt(p * (1.0 - p) / trials + z * z / (4.0 * trials * trials)) / den
    return centre - half, centre + half


def _quantile(values, q):
    v = np.sort(np.asarray(values, dtype=np.float64))
    if len(v) == 0:
        return None
    x = q * (len(v) - 1)
    lo, hi = int(math.floor(x)), int(math.ceil(x))
    return float(v[lo] + (x - lo) * (v[hi] - v[lo]))


def reference_gates(ref, other, min_events=30):
    """The reference's ensemble acceptance checks (validation/physics_validation.py:192-309),
    restated on engine results: 95 % capture intervals overlap, complete-evaporation fraction
    z <= 3, mean scatterings within 10 %, captured radial distribution total variation <= 0.10,
    evaporation-time median within 20 % and 90th percentile within 30 % (when both runs have
    at least `min_events` events).  Returns {name: (passed, value)}."""
    ca, cb = ref["counters"], other["counters"]
    out = {}
    ia = wilson_interval(ca["captured"], ca["trajectories"])
    ib = wilson_interval(cb["captured"], cb["trajectories"])
    out["capture_95pct_intervals_overlap"] = (max(ia[0], ib[0]) <= min(ia[1], ib[1]), [ia, ib])
    ea, eb = len(ref["events"]), len(other["events"])
    na, nb = ca["captured"], cb["captured"]
    if na > 0 and nb > 0:
        pooled = (ea + eb) / (na + nb)
        var = pooled * (1.0 - pooled) * (1.0 / na + 1.0 / nb)
        diff = abs(ea / na - eb / nb)
        z = (0.0 if diff == 0.0 else math.inf) if var <= 0.0 else diff / math.sqrt(var)
        out["complete_evaporation_fraction_z"] = (z <= 3.0, z)
    sa = ca["total_scatterings"] / max(ca["trajectories"], 1)
    sb = cb["total_scatterings"] / max(cb["trajectories"], 1)
    d = abs(sb - sa) / max(abs(sa), 1.0)
    out["average_scatterings_relative_difference"] = (d <= 0.10, d)
    ha = np.asarray(ref["histograms"][HIST_CAPTURED_DT], dtype=np.float64)
    hb = np.asarray(other["histograms"][HIST_CAPTURED_DT], dtype=np.float64)
    if ha.sum() > 0 and hb.sum() > 0:
        tv = 0.5 * float(np.sum(np.abs(hb / hb.sum() - ha / ha.sum())))
        out["captured_radial_total_variation"] = (tv <= 0.10, tv)
    if ea >= min_events and eb >= min_events:
        la, lb = ref["events"]["lifetime_unbinding"], other["events"]["lifetime_unbinding"]
        for name, q, limit in (("evaporation_median_relative_difference", 0.5, 0.20),
                               ("evaporation_p90_relative_difference", 0.9, 0.30)):
            qa, qb = _quantile(la, q), _quantile(lb, q)
            d = abs(qb - qa) / max(abs(qa), 1.0e-300)
            out[name] = (d <= limit, d)
    return out


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
