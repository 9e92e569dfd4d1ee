/*
 * dms_constants.h — physical constants, unit conventions and algorithm constants of the
 * DaMaSCUS-SUN trajectory Monte Carlo, shared by the CUDA engine, the host library and the
 * CPU oracle so that every implementation starts from identical numbers.
 *
 * Unit system of the engine (device and host tables): km, s, km/s, eV for energies,
 * Kelvin for temperatures, 1/km^3 for number densities, km^2 for cross sections and 1/s for
 * scattering rates.  The reference computes in natural units (hbar = c = 1, GeV); the factors
 * below convert between the two.  G*M_sun in natural units (~7e-39 GeV^-2 times a huge mass)
 * is subnormal-prone in FP32, which is one reason the engine works in km/s instead.
 *
 * Plain C99 preprocessor constants: usable from C, C++ and CUDA.
 */
#ifndef DMS_CONSTANTS_H
#define DMS_CONSTANTS_H

/* --- fundamental constants (CODATA 2018 / IAU 2015 nominal values) --------------------- */
#define DMS_C_KMS            299792.458              /* speed of light [km/s] */
#define DMS_HBAR_GEV_S       6.582119569e-25         /* hbar [GeV s] */
#define DMS_HBARC_GEV_M      1.973269804e-16         /* hbar*c [GeV m] */
#define DMS_GEV_PER_KG       5.609588603804452e26    /* c^2 / (1e9 e) [GeV/kg] */
#define DMS_KB_GEV_PER_K     8.617333262e-14         /* Boltzmann constant [GeV/K] */
#define DMS_G_SI             6.67430e-11             /* Newton constant [m^3 kg^-1 s^-2] */
#define DMS_MSUN_KG          1.98841e30              /* solar mass [kg] (IAU GM_sun / G) */
#define DMS_RSUN_KM          6.957e5                 /* solar radius [km]; the reference's
                                                        R_SUN_KM, include/Simulation_Trajectory.hpp:28 */
#define DMS_AU_KM            1.495978707e8           /* astronomical unit [km] */
#define DMS_MPROTON_GEV      0.93827208816           /* proton mass [GeV] */
#define DMS_MELECTRON_GEV    0.51099895000e-3        /* electron mass [GeV] */
#define DMS_MNUCLEON_GEV     0.93149410242           /* atomic mass unit [GeV]; isotope mass = A*u */
#define DMS_ALPHA_EM         (1.0 / 137.035999084)   /* fine-structure constant (CODATA 2018) */

/* G*M_sun [km^3/s^2]; the engine stores G*M(r) directly (gravitational parameter). */
#define DMS_GMSUN_KM3S2      (DMS_G_SI * DMS_MSUN_KG * 1.0e-9)

/* --- reference algorithm constants (src/Simulation_Trajectory.cpp:29-43, 53-81) ---------- */
#define DMS_RK45_MIN_STEP_FACTOR        0.1
#define DMS_RK45_MAX_STEP_FACTOR        4.0
#define DMS_RK45_MAX_INNER_RETRIES      256
#define DMS_RK45_ABS_MAX_STEP_S         1.0e6      /* RK45_Absolute_Max_Time_Step */
#define DMS_RK45_ABS_MIN_STEP_S         1.0e-8     /* abs_min_step, :1570 */
#define DMS_RK45_DEFAULT_STEP_S         0.1        /* RK45_Sanitized_Time_Step fallback */
#define DMS_RK45_TOL_R_KM               1.0        /* error_tolerances, :1461-1463 */
#define DMS_RK45_TOL_V_KMS              1.0e-3
#define DMS_RK45_TOL_PHI                1.0e-7
#define DMS_FREE_ENERGY_DRIFT_REL_E_SCALE_EV 1.0e-30
#define DMS_MAX_OPTICAL_DEPTH_STEP      0.05
#define DMS_CAPTURE_MAX_OPTICAL_DEPTH_STEP 0.10
#define DMS_OPTICAL_DEPTH_REL_TOL       1.0e-2
#define DMS_OPTICAL_DEPTH_ABS_TOL       (1.0e-12 * DMS_MAX_OPTICAL_DEPTH_STEP)
#define DMS_MAX_OPTICAL_DEPTH_RETRIES   100
#define DMS_MAX_OPTICAL_DEPTH_PIECES    4
#define DMS_CAPTURE_OPTICAL_DEPTH_PIECES 2
#define DMS_TARGET_VELOCITY_MAX_REJECTIONS 10000UL
#define DMS_V_MAX_C                     0.75       /* v_max of Trajectory_Simulator and of the rate grid */
#define DMS_KEPLER_DOMAIN_TOLERANCE     1.0e-10    /* src/Simulation_Utilities.cpp:22 */

/* --- radial bincount (include/Simulation_Trajectory.hpp:27-30) --------------------------- */
#define DMS_NUM_BINS                    2000
#define DMS_BIN_MAX_KM                  (2.0 * DMS_RSUN_KM)
#define DMS_BIN_WIDTH_KM                (DMS_BIN_MAX_KM / DMS_NUM_BINS)

/* --- initial conditions (src/Simulation_Utilities.cpp:186, 220) -------------------------- */
#define DMS_IC_SPEED_YMAX_NATURAL       1200.0     /* rejection y_max, natural units (1/c) */
#define DMS_IC_ASYMPTOTIC_DISTANCE_AU   1000.0

/* --- solar model ------------------------------------------------------------------------ */
#define DMS_SOLAR_DATA_SKIP_LINES       20         /* src/Solar_Model.cpp:46 */
#define DMS_SOLAR_COLUMNS               35
#define DMS_SOLAR_ELEMENT_COLUMNS       29         /* H1 ... Ni, columns 7-35 of the file */
#define DMS_PHOTOSPHERE_T_K             5800.0     /* src/Solar_Model.cpp:58 */
#define DMS_PHOTOSPHERE_RHO_GCM3        1.0e-9     /* src/Solar_Model.cpp:60 */

#endif /* DMS_CONSTANTS_H */
