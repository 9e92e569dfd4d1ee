/*
 * dms_philox.h — the engine's random-draw stream.
 *
 * Every uniform draw of a trajectory is a pure function of
 *     (seed, parameter point, trajectory id, draw index)
 * so any trajectory can be replayed on the CPU or the GPU, in any order, by any number of
 * threads.  The generator is Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11), restated from the published round function:
 *     key    = (seed, point)
 *     counter= (draw index low 32 bits, draw index high 32 bits, trajectory low, trajectory high)
 * Output words 0 and 1 form one double with 53 random bits in [0, 1); words 2 and 3 are
 * unused so that draw n depends on nothing but n.
 *
 * The reference draws through std::mt19937 + libphysica::Sample_Uniform
 * (src/Simulation_Trajectory.cpp:103-107, 795, 1144, 1193-1219, 1238); the engine keeps the
 * reference's draw ORDER and COUNT per function and replaces only the bit source.
 */
#ifndef DMS_PHILOX_H
#define DMS_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define DMS_HD __host__ __device__ __forceinline__
#else
#define DMS_HD static inline
#endif

#define DMS_PHILOX_M0 0xD2511F53u
#define DMS_PHILOX_M1 0xCD9E8D57u
#define DMS_PHILOX_W0 0x9E3779B9u
#define DMS_PHILOX_W1 0xBB67AE85u

DMS_HD void dms_philox_mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo)
{
	const uint64_t p = (uint64_t)a * (uint64_t)b;
	*hi = (uint32_t)(p >> 32);
	*lo = (uint32_t)p;
}

/* Philox4x32 with 10 rounds: ctr[4], key[2] -> out[4]. */
DMS_HD void dms_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
	uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
	uint32_t k0 = key[0], k1 = key[1];
	for(int round = 0; round < 10; round++)
	{
		uint32_t hi0, lo0, hi1, lo1;
		dms_philox_mulhilo(DMS_PHILOX_M0, c0, &hi0, &lo0);
		dms_philox_mulhilo(DMS_PHILOX_M1, c2, &hi1, &lo1);
		const uint32_t n0 = hi1 ^ c1 ^ k0;
		const uint32_t n1 = lo1;
		const uint32_t n2 = hi0 ^ c3 ^ k1;
		const uint32_t n3 = lo0;
		c0 = n0;
		c1 = n1;
		c2 = n2;
		c3 = n3;
		k0 += DMS_PHILOX_W0;
		k1 += DMS_PHILOX_W1;
	}
	out[0] = c0;
	out[1] = c1;
	out[2] = c2;
	out[3] = c3;
}

/* Uniform double in [0, 1) with 53 random bits. */
DMS_HD double dms_draw_uniform(uint32_t seed, uint32_t point, uint64_t trajectory, uint64_t draw_index)
{
	uint32_t ctr[4], key[2], out[4];
	ctr[0] = (uint32_t)draw_index;
	ctr[1] = (uint32_t)(draw_index >> 32);
	ctr[2] = (uint32_t)trajectory;
	ctr[3] = (uint32_t)(trajectory >> 32);
	key[0] = seed;
	key[1] = point;
	dms_philox4x32_10(ctr, key, out);
	const double hi = (double)(out[0] >> 5);   /* 27 bits */
	const double lo = (double)(out[1] >> 6);   /* 26 bits */
	return (hi * 67108864.0 + lo) * (1.0 / 9007199254740992.0);
}

#endif /* DMS_PHILOX_H */
