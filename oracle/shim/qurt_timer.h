/* Build shim (test infrastructure only). */
#ifndef ROVER_SHIM_QURT_TIMER_H
#define ROVER_SHIM_QURT_TIMER_H
#include "qurt.h"
int qurt_timer_sleep(unsigned long long duration_us);
#endif
