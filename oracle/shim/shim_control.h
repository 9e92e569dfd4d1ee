/* Oracle test shim: control of the draw stream used by the shimmed libphysica sampling
 * functions.  A stream is the engine's Philox stream keyed by (seed, point, trajectory);
 * dms_shim_set_stream() selects it and resets the draw index to 0. */
#ifndef DMS_SHIM_CONTROL_H
#define DMS_SHIM_CONTROL_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
void dms_shim_set_stream(uint32_t seed, uint32_t point, uint64_t trajectory);
uint64_t dms_shim_draw_count(void);
void dms_shim_set_tracing(int on);
size_t dms_shim_trace_size(void);
const double* dms_shim_trace_data(void);
#ifdef __cplusplus
}
#endif
#endif
