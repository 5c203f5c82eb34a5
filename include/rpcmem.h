/*
 * rpcmem.h -- shared-buffer allocator of the FastRPC host library, as
 * exported by libcalculator.so for hosts that drive the *_dma entry points
 * (the reference host calls these from retrieval_rpc_demo_pipeline.c and
 * retrieval_rpc_demo_pure_pq.c).  Buffers are pinned host memory; the "fd"
 * of a buffer names it in the *_dma calls.
 */
#ifndef ROVER_RPCMEM_H
#define ROVER_RPCMEM_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
#define RPCMEM_HEAP_ID_SYSTEM 25
#define RPCMEM_DEFAULT_FLAGS 1
#define RPCMEM_FLAG_UNCACHED 0
void rpcmem_init(void);
void rpcmem_deinit(void);
void *rpcmem_alloc(int heapid, uint32_t flags, int size);
void rpcmem_free(void *po);
int rpcmem_to_fd(void *po);
#ifdef __cplusplus
}
#endif
#endif
