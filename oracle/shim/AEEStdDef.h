/* Build shim (test infrastructure only): the Hexagon SDK scalar typedefs the
 * reference sources use, restated for an x86-64 host build of the oracle. */
#ifndef ROVER_SHIM_AEESTDDEF_H
#define ROVER_SHIM_AEESTDDEF_H
#include <stdint.h>
typedef int32_t int32;
typedef uint32_t uint32;
typedef int16_t int16;
typedef uint16_t uint16;
typedef int8_t int8;
typedef uint8_t uint8;
typedef int64_t int64;
typedef uint64_t uint64;
typedef int AEEResult;
#endif
