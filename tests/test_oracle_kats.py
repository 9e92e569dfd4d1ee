"""The oracle against the reference's own known-answer tests (tests/test_Solar_Model.cpp,
tests/test_Physics_Validation.cpp of the reference) and the draw-stream / math building blocks."""
import ctypes
import math

import numpy as np
import pytest

from dms_ctypes import C_KMS, NUM_TARGETS, RSUN_KM, point_params

GMSUN = 6.67430e-11 * 1.98841e30 * 1e-9
KB = 8.617333262e-14
MP = 0.93827208816


def test_escape_speed_kats(oracle):
    # tests/test_Solar_Model.cpp:73-81
    assert abs(oracle.query(2, 0.0) - 1384.13) < 0.1
    assert oracle.query(2, RSUN_KM) == pytest.approx(math.sqrt(2 * GMSUN / RSUN_KM), rel=4e-16)
    assert oracle.query(2, 2 * RSUN_KM) == pytest.approx(math.sqrt(2 * GMSUN / 2 / RSUN_KM), rel=4e-16)


def test_temperature_kats(oracle):
    # tests/test_Solar_Model.cpp:63-71 (1e-20 GeV tolerance at R_sun)
    assert oracle.query(1, 0.0) == pytest.approx(1.549e7, rel=4e-16)
    assert abs(oracle.query(1, RSUN_KM) - 5800.0) < 1e-20 / KB
    assert oracle.query(1, 0.96950 * RSUN_KM) == pytest.approx(1.544e5, rel=4e-16)


def test_mass_kats(oracle):
    # tests/test_Solar_Model.cpp:53-61
    assert oracle.query(0, 0.0) == 0.0
    assert oracle.query(0, RSUN_KM) == pytest.approx(GMSUN, rel=4e-16)
    assert oracle.query(0, 0.00150 * RSUN_KM) == pytest.approx(4e-7 * GMSUN, rel=4e-16)


def test_hydrogen_density_kat(oracle):
    # tests/test_Solar_Model.cpp:30-41: n_H1 = 0.36209 * 150.5 g/cm^3 / m_p, flat inside 0.0015 R_sun
    m_kg = MP / 5.609588603804452e26
    n_h1 = 0.36209 * 1.505e2 * 1e12 / m_kg
    for r in (0.0, 0.001 * RSUN_KM, 0.0015 * RSUN_KM):
        assert oracle.query(4, r, 0) == pytest.approx(n_h1, rel=4e-16)


def test_electron_density_is_charge_weighted_sum(oracle):
    # tests/test_Solar_Model.cpp:99-110
    from dms_ctypes import Oracle  # noqa: F401
    zs = [1, 2, 2, 6, 6, 7, 7, 8, 8, 8] + [10] * 3 + [11] + [12] * 3 + [13] + [14] * 3 + [15] + [16] * 4 + [17] * 2 + \
         [18] * 3 + [19] * 3 + [20] * 6 + [21] + [22] * 5 + [23] * 2 + [24] * 4 + [25] + [26] * 4 + [27] + [28] * 5
    assert len(zs) == NUM_TARGETS
    r = 0.5 * RSUN_KM
    ne = sum(z * oracle.query(4, r, i) for i, z in enumerate(zs))
    assert oracle.query(3, r) == pytest.approx(ne, rel=1e-14)
    assert oracle.query(3, 1.5 * RSUN_KM) == 0.0


def test_thermal_relative_speed_kat(oracle):
    # tests/test_Solar_Model.cpp:267-281 (speeds in units of c there)
    v = 1e-3 * C_KMS
    assert abs(oracle.query(7, 1e7, MP, v) / C_KMS - 0.0017928) < 1e-7
    assert abs(oracle.query(7, 0.01, MP, v) / C_KMS - 1e-3) < 1e-10
    zero = oracle.query(7, 1e7, MP, 0.0)
    assert math.isfinite(zero) and zero > 0.0
    assert math.isnan(oracle.query(7, 0.0, MP, v))
    assert math.isnan(oracle.query(7, 1e7, MP, -v))


def test_maxwell_mean_speed_limit(oracle):
    # tests/test_Physics_Validation.cpp:232-240: <v_rel>(v=0) = sqrt(8T/(pi m)) to 1e-12
    T, m = 1.2e7, 4 * 0.93149410242
    expect = math.sqrt(8 * T * KB / (math.pi * m)) * C_KMS
    assert oracle.query(7, T, m, 0.0) == pytest.approx(expect, rel=1e-12)


@pytest.fixture(scope="module")
def oracle_point(oracle):
    oracle.set_point(point_params(0.01, 1e-36, sigma_e_cm2=0.0, interpolation_points=1000))
    return oracle


def test_total_rate_is_sum_of_channels(oracle_point):
    # tests/test_Solar_Model.cpp:145-166
    r, v = 0.5 * RSUN_KM, 1e-3 * C_KMS
    total = oracle_point.query(12, r, -1, v) + sum(oracle_point.query(12, r, i, v) for i in range(NUM_TARGETS))
    assert oracle_point.query(6, r, v) == pytest.approx(total, rel=4e-16)
    assert oracle_point.query(5, 1.5 * RSUN_KM, v) == 0.0


def test_interpolated_rate_within_10_percent(oracle_point):
    # tests/test_Solar_Model.cpp:168-190: m = 0.01 GeV, sigma = 1 pb, 1000^2 grid, 500 samples, w <= 0.3 c
    rng = np.random.default_rng(998)
    for _ in range(500):
        r = rng.uniform(0, RSUN_KM)
        w = rng.uniform(0, 0.3) * C_KMS
        exact = oracle_point.query(6, r, w)
        assert abs(oracle_point.query(5, r, w) - exact) <= 0.1 * exact


def test_grid_nodes_exact(oracle):
    # tests/test_Solar_Model.cpp:192-225 (square grid: the engine builds N x N as src/main.cpp:80)
    N = 31
    oracle.set_point(point_params(0.01, 1e-36, sigma_e_cm2=0.0, interpolation_points=N))
    for i in (0, 7, 15, 30):
        for j in (0, 5, 14, 28):
            r = RSUN_KM * i / (N - 1)
            v = 0.75 * j / (N - 1) * C_KMS
            exact = oracle.query(6, r, v)
            # the reference's floor is 1e-30 in natural units (GeV); 1 GeV = 1/hbar [1/s]
            floor = 1e-30 / 6.582119569e-25
            assert abs(oracle.query(5, r, v) - exact) <= max(floor, 1e-10 * abs(exact))
    assert math.isnan(oracle.query(5, float("nan"), 300.0))
    assert math.isnan(oracle.query(5, 0.5 * RSUN_KM, float("nan")))


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    import os
    import subprocess
    import tempfile
    from dms_ctypes import REPO
    src = r'''
#include <stdio.h>
#include "dms_philox.h"
int main(void){
  uint32_t c0[4]={0,0,0,0}, k0[2]={0,0}, o[4];
  dms_philox4x32_10(c0,k0,o); printf("%08x %08x %08x %08x\n",o[0],o[1],o[2],o[3]);
  uint32_t c1[4]={0xffffffffu,0xffffffffu,0xffffffffu,0xffffffffu}, k1[2]={0xffffffffu,0xffffffffu};
  dms_philox4x32_10(c1,k1,o); printf("%08x %08x %08x %08x\n",o[0],o[1],o[2],o[3]);
  uint32_t c2[4]={0x243f6a88u,0x85a308d3u,0x13198a2eu,0x03707344u}, k2[2]={0xa4093822u,0x299f31d0u};
  dms_philox4x32_10(c2,k2,o); printf("%08x %08x %08x %08x\n",o[0],o[1],o[2],o[3]);
  return 0; }
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "kat.c")
        exe = os.path.join(d, "kat")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-O2", "-I", os.path.join(REPO, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    assert out[0] == "6627e8d5 e169c58d bc57ac4c 9b00dbd8"
    assert out[1] == "408f276d 41c83b0e a20bc7c6 6d5451fd"
    assert out[2] == "d16cfe09 94fdcceb 5001e420 24126ea1"


def test_direct_rate_point_uses_the_computed_rate(oracle):
    """interpolation_points < 2 builds no grid: every lookup is the 64-channel sum
    (Interpolate_Total_DM_Scattering_Rate with N < 2, src/Solar_Model.cpp:397-405)."""
    import dms_ctypes
    oracle.set_point(dms_ctypes.point_params(0.3, 1e-36, interpolation_points=0))
    for r, v in ((1.0e4, 300.0), (3.0e5, 900.0), (6.9e5, 1500.0)):
        assert oracle.query(5, r, v) == oracle.query(6, r, v) > 0.0
    recs = oracle.run_records(7, 0, 0, 8, capture_mode=True, max_scatterings=10 ** 5)["records"]
    assert all(recs[i].termination_reason in range(11) for i in range(8))
