// Counters of the op-counting oracle build (see opcount.hpp).
#include <cstdint>

namespace dms_ops
{
uint64_t ops[4][5] = {};
uint64_t units[4] = {0, 0, 0, 0};
int phase = 3;
}	// namespace dms_ops

// out[24]: ops[phase][class] (20 values, phase-major), then units: attempts, steps,
// scatterings, trajectories
extern "C" void dms_opcount_get(uint64_t* out)
{
	for(int p = 0; p < 4; p++)
		for(int c = 0; c < 5; c++) out[5 * p + c] = dms_ops::ops[p][c];
	for(int k = 0; k < 4; k++) out[20 + k] = dms_ops::units[k];
}

extern "C" void dms_opcount_reset(void)
{
	for(int p = 0; p < 4; p++)
		for(int c = 0; c < 5; c++) dms_ops::ops[p][c] = 0;
	for(int k = 0; k < 4; k++) dms_ops::units[k] = 0;
	dms_ops::phase = 3;
}
