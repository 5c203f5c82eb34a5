/* Build shim (test infrastructure only): fd -> mapping lookup served by the
 * rpcmem registry in oracle/shim/shim.c. */
#ifndef ROVER_SHIM_HAP_MEM_H
#define ROVER_SHIM_HAP_MEM_H
#include <stdint.h>
#include "AEEStdDef.h"
int HAP_mmap_get(int fd, void **vaddr, uint64 *paddr);
int HAP_mmap_put(int fd);
#endif
