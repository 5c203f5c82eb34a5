/*
 * remote.h -- the FastRPC session calls the reference host makes
 * (src/app/main.c:13-20, retrieval_rpc_demo_pure_pq.c:80-127), exported by
 * libcalculator.so.  On a GPU there is no remote process: the calls
 * validate their arguments and record mappings of rpcmem buffers.
 */
#ifndef ROVER_REMOTE_H
#define ROVER_REMOTE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef uint64_t remote_handle64;
#define DSPRPC_CONTROL_UNSIGNED_MODULE 2
struct remote_rpc_control_unsigned_module { int domain; int enable; };
int remote_session_control(uint32_t req, void *data, uint32_t datalen);
enum fastrpc_map_flags { FASTRPC_MAP_STATIC = 0, FASTRPC_MAP_RESERVED = 1, FASTRPC_MAP_FD = 2 };
int fastrpc_mmap(int domain, int fd, void *addr, int offset, size_t length, enum fastrpc_map_flags flags);
int fastrpc_munmap(int domain, int fd, void *addr, size_t length);
#ifdef __cplusplus
}
#endif
#endif
