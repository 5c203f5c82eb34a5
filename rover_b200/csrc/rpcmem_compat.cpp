// rpcmem_compat.cpp -- rpcmem / fastrpc host calls exported by
// libcalculator.so.  A buffer is pinned host memory (cudaHostAlloc) named by
// an integer "fd"; the *_dma entry points resolve fds through
// rover_rpcmem_lookup and upload the contents to the device.
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/remote.h"
#include "../../include/rpcmem.h"
#include "rpcmem_compat.h"

namespace {
struct Buffer { void* ptr = nullptr; size_t size = 0; bool pinned = false; bool live = false; };
constexpr int kFdBase = 1000;
std::mutex g_lock;
std::vector<Buffer> g_buffers;
}  // namespace

extern "C" void rpcmem_init(void) {}
extern "C" void rpcmem_deinit(void) {}

extern "C" void* rpcmem_alloc(int heapid, uint32_t flags, int size) {
  (void)heapid; (void)flags;
  if (size <= 0) return nullptr;
  Buffer b;
  b.size = static_cast<size_t>(size);
  if (cudaHostAlloc(&b.ptr, b.size, cudaHostAllocPortable) == cudaSuccess) {
    b.pinned = true;
  } else {
    cudaGetLastError();
    b.ptr = std::malloc(b.size);
    if (!b.ptr) return nullptr;
  }
  b.live = true;
  std::lock_guard<std::mutex> lock(g_lock);
  for (auto& slot : g_buffers)
    if (!slot.live) { slot = b; return b.ptr; }
  g_buffers.push_back(b);
  return b.ptr;
}

extern "C" void rpcmem_free(void* po) {
  if (!po) return;
  Buffer b;
  {
    std::lock_guard<std::mutex> lock(g_lock);
    for (auto& slot : g_buffers)
      if (slot.live && slot.ptr == po) { b = slot; slot = Buffer(); break; }
  }
  if (!b.live) return;
  if (b.pinned) cudaFreeHost(b.ptr); else std::free(b.ptr);
}

extern "C" int rpcmem_to_fd(void* po) {
  std::lock_guard<std::mutex> lock(g_lock);
  for (size_t i = 0; i < g_buffers.size(); ++i)
    if (g_buffers[i].live && g_buffers[i].ptr == po) return kFdBase + static_cast<int>(i);
  return -1;
}

int rover_rpcmem_lookup(int fd, void** ptr, size_t* bytes) {
  std::lock_guard<std::mutex> lock(g_lock);
  const long i = static_cast<long>(fd) - kFdBase;
  if (i < 0 || i >= static_cast<long>(g_buffers.size()) || !g_buffers[i].live) return -1;
  if (ptr) *ptr = g_buffers[i].ptr;
  if (bytes) *bytes = g_buffers[i].size;
  return 0;
}

extern "C" int fastrpc_mmap(int domain, int fd, void* addr, int offset, size_t length, enum fastrpc_map_flags flags) {
  (void)domain; (void)flags;
  void* p = nullptr;
  size_t n = 0;
  if (rover_rpcmem_lookup(fd, &p, &n) != 0 || p != addr || offset < 0 ||
      static_cast<size_t>(offset) + length > n)
    return -1;
  return 0;
}

extern "C" int fastrpc_munmap(int domain, int fd, void* addr, size_t length) {
  (void)domain; (void)addr; (void)length;
  return rover_rpcmem_lookup(fd, nullptr, nullptr) == 0 ? 0 : -1;
}

extern "C" int remote_session_control(uint32_t req, void* data, uint32_t datalen) {
  (void)req;
  return (data || datalen == 0) ? 0 : -1;
}
