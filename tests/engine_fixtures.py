"""Shared helpers for tests that drive the CUDA engine through its C ABI."""
import os
import sys

from dms_ctypes import PACKAGE_DIR

if PACKAGE_DIR not in sys.path:
    sys.path.insert(0, PACKAGE_DIR)

import dms_b200  # noqa: E402

REPLAY_POINT = dict(mass_gev=0.3, sigma_p_cm2=1e-36, interpolation_points=200)


def outcome(rec):
    return (rec.number_of_scatterings, rec.termination_reason, rec.flags, rec.number_of_draws)


def state(rec):
    return [rec.final_time] + list(rec.final_position) + list(rec.final_velocity)
