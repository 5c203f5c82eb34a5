/* Build shim (test infrastructure only): DSP logging compiled out unless
 * ROVER_SHIM_FARF is defined. */
#ifndef ROVER_SHIM_HAP_FARF_H
#define ROVER_SHIM_HAP_FARF_H
#include <stdio.h>
#ifdef ROVER_SHIM_FARF
#define FARF(level, ...) (fprintf(stderr, __VA_ARGS__), fputc('\n', stderr))
#else
#define FARF(level, ...) ((void)0)
#endif
#endif
