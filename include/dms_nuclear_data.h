/*
 * dms_nuclear_data.h — the solar scattering targets.
 *
 * The reference builds its target list in Solar_Model::Solar_Model()
 * (src/Solar_Model.cpp:143-163): ten single isotopes for the first ten mass-fraction
 * columns (H1, He4, He3, C12, C13, N14, N15, O16, O17, O18, each with abundance 1), then every
 * stable isotope of the elements Z = 10..28 weighted by its natural abundance.  The element
 * data come from obscura's nuclear data files, which are not part of the reference; this
 * table restates the IUPAC representative isotopic compositions of those elements.
 * Isotope masses follow one rule: m_proton for A = 1, A * u otherwise (u = DMS_MNUCLEON_GEV).
 *
 * Column of the AGSS09 file for target k: 6 + element index (0-based), see
 * Create_Number_Density_Table, src/Solar_Model.cpp:98-110.
 */
#ifndef DMS_NUCLEAR_DATA_H
#define DMS_NUCLEAR_DATA_H

typedef struct
{
	unsigned char element_index; /* 0..28: mass-fraction column index (file column 6 + index) */
	unsigned char Z;
	unsigned char A;
	double abundance;
} dms_target_isotope;

/* Number of targets: 10 single isotopes + 53 natural isotopes of Z = 10..28. */
#define DMS_NUM_TARGETS 63

static const dms_target_isotope DMS_TARGET_ISOTOPES[DMS_NUM_TARGETS] = {
	{0, 1, 1, 1.0},   /* H1  */
	{1, 2, 4, 1.0},   /* He4 */
	{2, 2, 3, 1.0},   /* He3 */
	{3, 6, 12, 1.0},  /* C12 */
	{4, 6, 13, 1.0},  /* C13 */
	{5, 7, 14, 1.0},  /* N14 */
	{6, 7, 15, 1.0},  /* N15 */
	{7, 8, 16, 1.0},  /* O16 */
	{8, 8, 17, 1.0},  /* O17 */
	{9, 8, 18, 1.0},  /* O18 */
	{10, 10, 20, 0.9048}, {10, 10, 21, 0.0027}, {10, 10, 22, 0.0925},                 /* Ne */
	{11, 11, 23, 1.0},                                                                 /* Na */
	{12, 12, 24, 0.7899}, {12, 12, 25, 0.1000}, {12, 12, 26, 0.1101},                 /* Mg */
	{13, 13, 27, 1.0},                                                                 /* Al */
	{14, 14, 28, 0.92223}, {14, 14, 29, 0.04685}, {14, 14, 30, 0.03092},              /* Si */
	{15, 15, 31, 1.0},                                                                 /* P  */
	{16, 16, 32, 0.9499}, {16, 16, 33, 0.0075}, {16, 16, 34, 0.0425}, {16, 16, 36, 0.0001}, /* S */
	{17, 17, 35, 0.7576}, {17, 17, 37, 0.2424},                                        /* Cl */
	{18, 18, 36, 0.003336}, {18, 18, 38, 0.000629}, {18, 18, 40, 0.996035},           /* Ar */
	{19, 19, 39, 0.932581}, {19, 19, 40, 0.000117}, {19, 19, 41, 0.067302},           /* K  */
	{20, 20, 40, 0.96941}, {20, 20, 42, 0.00647}, {20, 20, 43, 0.00135},
	{20, 20, 44, 0.02086}, {20, 20, 46, 0.00004}, {20, 20, 48, 0.00187},              /* Ca */
	{21, 21, 45, 1.0},                                                                 /* Sc */
	{22, 22, 46, 0.0825}, {22, 22, 47, 0.0744}, {22, 22, 48, 0.7372},
	{22, 22, 49, 0.0541}, {22, 22, 50, 0.0518},                                        /* Ti */
	{23, 23, 50, 0.0025}, {23, 23, 51, 0.9975},                                        /* V  */
	{24, 24, 50, 0.04345}, {24, 24, 52, 0.83789}, {24, 24, 53, 0.09501}, {24, 24, 54, 0.02365}, /* Cr */
	{25, 25, 55, 1.0},                                                                 /* Mn */
	{26, 26, 54, 0.05845}, {26, 26, 56, 0.91754}, {26, 26, 57, 0.02119}, {26, 26, 58, 0.00282}, /* Fe */
	{27, 27, 59, 1.0},                                                                 /* Co */
	{28, 28, 58, 0.68077}, {28, 28, 60, 0.26223}, {28, 28, 61, 0.011399},
	{28, 28, 62, 0.036346}, {28, 28, 64, 0.009255},                                   /* Ni */
};

#endif /* DMS_NUCLEAR_DATA_H */
