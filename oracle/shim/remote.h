/* Build shim (test infrastructure only): FastRPC host API surface used by
 * the reference host sources, implemented in-process by oracle/shim/shim.c. */
#ifndef ROVER_SHIM_REMOTE_H
#define ROVER_SHIM_REMOTE_H
#include <stddef.h>
#include <stdint.h>
#include "AEEStdDef.h"
typedef uint64_t remote_handle64;
#define DSPRPC_CONTROL_UNSIGNED_MODULE 2
struct remote_rpc_control_unsigned_module { int domain; int enable; };
int remote_session_control(uint32_t req, void *data, uint32_t datalen);
enum fastrpc_map_flags { FASTRPC_MAP_STATIC = 0, FASTRPC_MAP_RESERVED = 1,
                         FASTRPC_MAP_FD = 2 };
int fastrpc_mmap(int domain, int fd, void *addr, int offset, size_t length,
                 enum fastrpc_map_flags flags);
int fastrpc_munmap(int domain, int fd, void *addr, size_t length);
#endif
