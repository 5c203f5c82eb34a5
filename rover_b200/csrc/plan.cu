// plan.cu -- the bookkeeping kernels of a search plan.
//
// A plan (calculator.cu) enqueues the same searches on every launch, so that
// a CUDA graph captured from one launch replays them on new query vectors.
// Host code cannot run between replays; what changes from launch to launch
// is kept on the device in PlanControl and updated by these two kernels, one
// before the searches and one after them.

#include "kernels.h"

namespace rover {

__global__ void __launch_bounds__(256) plan_prepare_kernel(PlanControl* ctl, unsigned long long* visited,
                                                           size_t visited_words, int32_t* status, int nq,
                                                           int classes) {
  const size_t tid = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  if (tid < static_cast<size_t>(classes)) ctl->counters[tid] = 0u;
  for (size_t i = tid; i < static_cast<size_t>(nq); i += stride) status[i] = 0;
  // ctl->clear is written only by plan_advance_kernel, which runs after the
  // searches: every block reads the same value here.
  if (*reinterpret_cast<volatile uint32_t*>(&ctl->clear)) {
    ulonglong2* v2 = reinterpret_cast<ulonglong2*>(visited);
    const size_t pairs = visited_words / 2;
    for (size_t i = tid; i < pairs; i += stride) v2[i] = make_ulonglong2(0ull, 0ull);
    if ((visited_words & 1) && tid == 0) visited[visited_words - 1] = 0ull;
  }
}

__global__ void plan_advance_kernel(PlanControl* ctl, int nq) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint64_t next = static_cast<uint64_t>(ctl->gen) + static_cast<uint64_t>(nq);
  if (next + static_cast<uint64_t>(nq) > 0xffffffffull) {
    // the tags of the next launch would wrap: restart at 1 on cleared tables
    ctl->gen = 1u;
    ctl->clear = 1u;
  } else {
    ctl->gen = static_cast<uint32_t>(next);
    ctl->clear = 0u;
  }
}

void launch_plan_prepare(PlanControl* ctl, unsigned long long* visited, size_t visited_words, int32_t* status, int nq,
                         int classes, int sms, cudaStream_t s) {
  // one wave of 4 blocks per SM: enough to zero gigabytes of tables at HBM
  // speed on the rare launch that clears, and a few microseconds otherwise
  plan_prepare_kernel<<<4 * sms, 256, 0, s>>>(ctl, visited, visited_words, status, nq, classes);
}

void launch_plan_advance(PlanControl* ctl, int nq, cudaStream_t s) { plan_advance_kernel<<<1, 32, 0, s>>>(ctl, nq); }

}  // namespace rover
