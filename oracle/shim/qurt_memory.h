/* Build shim (test infrastructure only): cache maintenance is a full memory
 * fence on a coherent host. */
#ifndef ROVER_SHIM_QURT_MEMORY_H
#define ROVER_SHIM_QURT_MEMORY_H
#include <stdint.h>
typedef uintptr_t qurt_addr_t;
typedef size_t qurt_size_t;
typedef enum { QURT_MEM_CACHE_FLUSH, QURT_MEM_CACHE_INVALIDATE,
               QURT_MEM_CACHE_FLUSH_INVALIDATE } qurt_mem_cache_op_t;
typedef enum { QURT_MEM_ICACHE, QURT_MEM_DCACHE } qurt_mem_cache_type_t;
int qurt_mem_cache_clean(qurt_addr_t addr, qurt_size_t size,
                         qurt_mem_cache_op_t op, qurt_mem_cache_type_t type);
#endif
