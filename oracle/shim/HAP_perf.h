/* Build shim (test infrastructure only). */
#ifndef ROVER_SHIM_HAP_PERF_H
#define ROVER_SHIM_HAP_PERF_H
#include <stdint.h>
uint64_t HAP_perf_get_time_us(void);
#endif
