// rpcmem_compat.h -- fd registry behind the exported rpcmem_* calls.
#pragma once
#include <cstddef>
// Resolve an rpcmem fd to its host pointer and size; 0 on success.
int rover_rpcmem_lookup(int fd, void** ptr, size_t* bytes);
