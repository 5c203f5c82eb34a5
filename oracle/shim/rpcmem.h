/* Build shim (test infrastructure only): rpcmem allocator as plain heap
 * memory plus an fd registry (oracle/shim/shim.c). */
#ifndef ROVER_SHIM_RPCMEM_H
#define ROVER_SHIM_RPCMEM_H
#include <stdint.h>
#define RPCMEM_HEAP_ID_SYSTEM 25
#define RPCMEM_DEFAULT_FLAGS 1
#define RPCMEM_FLAG_UNCACHED 0
void rpcmem_init(void);
void rpcmem_deinit(void);
void *rpcmem_alloc(int heapid, uint32_t flags, int size);
void rpcmem_free(void *po);
int rpcmem_to_fd(void *po);
#endif
