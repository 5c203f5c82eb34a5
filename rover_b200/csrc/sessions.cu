// sessions.cu -- the accelerator's lane-protocol sessions on a GPU.
//
// The reference host drives its pure-PQ and SQMD searches through shared
// memory (src/dsp_demo/retrieval_rpc_demo_pure_pq.c:80-190,
// retrieval_rpc_demo_pipeline.c:1298-1417): it allocates a control block
// with rpcmem_alloc, starts one blocking session call on a thread of its
// own, and then, query after query, writes neighbour ids into lane buffers,
// marks them CPU_READY and polls for DSP_DONE, reading back one quantized
// distance per id.  On the phone, lane worker threads of the DSP skeleton
// serve the buffers (retrieval_async_dsp_search.c:1036-1182, :2134-2265).
//
// Here the session call is a service loop on the host thread that made it:
// each pass collects every ready buffer of every lane, gathers their ids
// into one list, runs the library's distance kernel for the whole list on
// the GPU (PQ: the ADC sums of pq_adc_kernel over the host's own lookup
// table; SQ: the L1 code distance of sq_coarse_kernel), and writes the
// results and states back.  No kernel ever waits on the host: every wait on
// a shared flag is a host-side poll, and a session whose host stops talking
// to it for longer than the idle limit ends with AEE_EFAILED instead of
// spinning for ever.
//
// The shared structures below restate the byte layout of the reference's
// search-branch build (retrieval_sqmd_pure_pq.h:57-163,
// retrieval_db_common.h:56-190; RETRIEVAL_ENABLE_FULL_BUILD off), because
// the host that fills them is the reference's own code; the static_asserts
// pin every offset the service touches.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/calculator.h"
#include "../../include/rover_b200.h"
#include "kernels.h"
#include "rpcmem_compat.h"
#include "session_bridge.h"

namespace rover {
namespace {

constexpr int kLanesMax = 8;          // PURE_PQ_SQMD_MAX_LANES, SQMD_DSP_LANES
constexpr int kBuffersPerLane = 2;    // PURE_PQ_SQMD_BUFFERS_PER_LANE, SQMD_BUFFERS_PER_LANE
constexpr int kItemsMax = 32;         // PURE_PQ_SQMD_MAX_WORK_ITEMS, SQMD_MAX_WORK_ITEMS
constexpr int kMaxDim = 1024;         // RETRIEVAL_ASYNC_DEMO_MAX_DIM

// ---- pure-PQ control block -------------------------------------------------
enum : int32_t { kPqEmpty = 0, kPqCpuReady = 1, kPqDspDone = 2 };
enum : int32_t { kPqIdle = 0, kPqRunning = 1, kPqDone = 2, kPqShutdown = 3, kPqAbort = 4 };

struct PqWork { int32_t neighbor_id, source_id; };
struct PqResult { int32_t neighbor_id, source_id; float distance; };

struct alignas(128) PqLaneBuffer {
  volatile int32_t state;
  int32_t turn_id, query_gen, work_count, result_count;
  PqWork work[kItemsMax];
  PqResult result[kItemsMax];
};
struct PqLane {
  PqLaneBuffer buffers[kBuffersPerLane];
  volatile int32_t dsp_active_buffer;
  volatile int32_t cpu_fill_buffer;
};
struct alignas(128) PqLutHeader {
  volatile int32_t query_gen, lut_gen;
  int32_t m, ks, lut_count;
  uint8_t index_uuid[16];
  uint8_t reserved[128 - 5 * 4 - 16];
};
struct PqStats {
  volatile uint64_t work_items, dsp_compute_us, dsp_wait_cpu_us, dsp_wait_polls, abort_count;
};
struct PqControl {
  volatile int32_t control_state;
  int32_t lane_count, turn_id;
  volatile int32_t query_gen;
  uint8_t reserved[128 - 4 * 4];
  PqLane lanes[kLanesMax];
  PqStats stats;
};
static_assert(sizeof(PqLaneBuffer) == 768 && offsetof(PqLaneBuffer, work) == 20 &&
              offsetof(PqLaneBuffer, result) == 276, "pure-PQ lane buffer layout");
static_assert(sizeof(PqLane) == 1664 && offsetof(PqLane, dsp_active_buffer) == 1536, "pure-PQ lane layout");
static_assert(sizeof(PqLutHeader) == 128 && offsetof(PqLutHeader, index_uuid) == 20, "LUT header layout");
static_assert(offsetof(PqControl, lanes) == 128 && offsetof(PqControl, stats) == 128 + 8 * 1664 &&
              sizeof(PqControl) == 13568, "pure-PQ control layout");

// ---- SQMD control block ----------------------------------------------------
enum : int32_t { kSqEmpty = 0, kSqCpuReady = 1, kSqDspDone = 2, kSqDspAbort = 3 };
enum : int32_t { kCtrlRunning = 0, kCtrlDone = 1, kCtrlAbort = 2, kCtrlPreparing = 3 };
enum : int32_t { kSessIdle = 0, kSessRunning = 1, kSessShutdown = 2, kSessAbort = 3 };
enum : int32_t { kSqStatusBadParam = -1, kSqStatusTooMuchWork = -3 };
enum : int32_t { kContractLegacy = 0, kContractAlignedU8 = 0x12020001 };

struct SqWork { int32_t neighbor_id, source_id; };
struct SqResult { int32_t neighbor_id, source_id; float coarse_dist; };
struct alignas(128) SqLaneBuffer {
  volatile int32_t state;
  int32_t turn_id, work_count, result_count;
  SqWork work[kItemsMax];
  SqResult result[kItemsMax];
};
struct SqLane {
  SqLaneBuffer buf[kBuffersPerLane];
  volatile int32_t dsp_active_buf;
  alignas(128) volatile int32_t cpu_fill_buf;
};
struct SqStats {
  volatile uint64_t work_items, dedup_skips, empty_turns, dsp_compute_us, cpu_correct_us, cpu_wait_dsp_us,
      dsp_wait_cpu_us, dsp_invalidate_us, lane_wait_us, dsp_done_batches, dsp_wait_poll_count, abort_count;
  volatile int32_t abort_fields[12];
  volatile uint64_t pipeline[5];
};
struct alignas(128) SqQuerySlot {
  volatile int32_t query_gen;
  int32_t query_dim, contract_id, reserved;
  uint8_t query_u8[kMaxDim];
  float query[kMaxDim];
};
struct alignas(128) SqStartupSlot {
  volatile int32_t cancel, acknowledged;
  uint8_t pad[128 - 8];
};
struct SqControl {
  volatile int32_t ctrl_state;
  int32_t lane_count, turn_id;
  volatile int32_t session_state;
  uint8_t pad[128 - 16];
  SqLane lanes[kLanesMax];
  SqStats stats;
  SqQuerySlot query_slot;
  SqStartupSlot startup_slot;
};
static_assert(sizeof(SqLaneBuffer) == 768 && offsetof(SqLaneBuffer, work) == 16 &&
              offsetof(SqLaneBuffer, result) == 272, "SQMD lane buffer layout");
static_assert(sizeof(SqLane) == 1792 && offsetof(SqLane, cpu_fill_buf) == 1664, "SQMD lane layout");
static_assert(sizeof(SqStats) == 184 && offsetof(SqStats, abort_fields) == 96, "SQMD stats layout");
static_assert(sizeof(SqQuerySlot) == 5248 && offsetof(SqQuerySlot, query) == 1040, "SQMD query slot layout");
static_assert(offsetof(SqControl, lanes) == 128 && offsetof(SqControl, stats) == 128 + 8 * 1792 &&
              offsetof(SqControl, query_slot) == 14720 && offsetof(SqControl, startup_slot) == 19968 &&
              sizeof(SqControl) == 20096, "SQMD control layout");


// ---- DB-pair expansion buffers ---------------------------------------------
enum : int32_t { kDbEmpty = 0, kDbDspDone = 1, kDbCpuDone = 2 };
struct DbExpansion {
  volatile int32_t state;
  int32_t count, finished, pad;
  int32_t neighbor_ids[kItemsMax];
  float coarse_dists[kItemsMax];
  float corrected_dists[kItemsMax];
};
struct DbSharedStats {
  volatile uint64_t dsp_wait_cpu_done_us, dsp_invalidate_us, dsp_wait_poll_count;
};
struct DbShared {
  DbExpansion buf[2];
  DbSharedStats stats;
};
static_assert(sizeof(DbExpansion) == 400 && offsetof(DbExpansion, corrected_dists) == 272, "expansion buffer layout");
static_assert(sizeof(DbShared) == 824, "DB-pair shared layout");

// ---- the GPU side of one service pass ---------------------------------------
//
// One device block per session: [offsets: 2 x int64][status: int32, padded to
// 16 bytes][out: float x kSlots][ids: int32 x kSlots], and its pinned host
// twin.  A pass copies offsets, status and ids up in one transfer, runs one
// distance kernel over the whole id list, and copies status and distances
// back in one transfer.
constexpr int kSlots = kLanesMax * kBuffersPerLane * kItemsMax;
constexpr size_t kOffOut = 32, kOffIds = kOffOut + 4 * kSlots, kBlockBytes = kOffIds + 4 * kSlots;

class GpuPass {
 public:
  ~GpuPass() { release(); }

  bool init(size_t table_floats) {
    table_floats_ = table_floats;
    if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&d_block_, kBlockBytes) != cudaSuccess ||
        cudaMalloc(&d_table_, table_floats * sizeof(float)) != cudaSuccess ||
        cudaHostAlloc(&h_block_, kBlockBytes, cudaHostAllocDefault) != cudaSuccess) {
      session_error("session set-up: %s", cudaGetErrorString(cudaGetLastError()));
      return false;
    }
    return true;
  }

  void release() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (d_block_) cudaFree(d_block_);
    if (d_table_) cudaFree(d_table_);
    if (h_block_) cudaFreeHost(h_block_);
    if (stream_) cudaStreamDestroy(stream_);
    d_block_ = d_table_ = nullptr;
    h_block_ = nullptr;
    stream_ = nullptr;
  }

  int32_t* ids() { return reinterpret_cast<int32_t*>(static_cast<uint8_t*>(h_block_) + kOffIds); }
  const float* out() const { return reinterpret_cast<const float*>(static_cast<const uint8_t*>(h_block_) + kOffOut); }

  // The per-query table: the PQ lookup table (m * ks floats), the FP32
  // query, or the aligned u8 query of the split distance (bytes).
  bool upload_table(const void* src, size_t bytes) {
    if (bytes > table_floats_ * sizeof(float)) return false;
    if (cudaMemcpyAsync(d_table_, src, bytes, cudaMemcpyHostToDevice, stream_) != cudaSuccess)
      return fail("table upload");
    return cudaStreamSynchronize(stream_) == cudaSuccess || fail("table upload");
  }

  // Distances of ids()[0, n): PQ ADC (pq != nullptr), or SQ L1 distance
  // (against the aligned u8 query when `aligned`).  False on a CUDA error or
  // a kernel-reported failure.
  bool run(const PqIndexView* pq, const SqIndexView* sq, int n, uint64_t* gpu_us, bool aligned = false) {
    const auto t0 = std::chrono::steady_clock::now();
    uint8_t* hb = static_cast<uint8_t*>(h_block_);
    int64_t* off = reinterpret_cast<int64_t*>(hb);
    off[0] = 0;
    off[1] = n;
    *reinterpret_cast<int32_t*>(hb + 16) = 0;
    // offsets, status and (the unused) out travel with the ids: one transfer
    if (cudaMemcpyAsync(d_block_, h_block_, kOffIds + 4u * n, cudaMemcpyHostToDevice, stream_) != cudaSuccess)
      return fail("id upload");
    uint8_t* db = static_cast<uint8_t*>(d_block_);
    const int64_t* d_off = reinterpret_cast<const int64_t*>(db);
    int32_t* d_status = reinterpret_cast<int32_t*>(db + 16);
    float* d_out = reinterpret_cast<float*>(db + kOffOut);
    const int32_t* d_ids = reinterpret_cast<const int32_t*>(db + kOffIds);
    if (pq) launch_pq_adc(*pq, d_table_, 1, d_ids, d_off, d_out, d_status, stream_);
    else if (aligned) launch_sq_aligned_coarse(*sq, reinterpret_cast<const uint8_t*>(d_table_), 1, d_ids, d_off, d_out,
                                               d_status, stream_);
    else launch_sq_coarse(*sq, d_table_, 1, d_ids, d_off, d_out, d_status, stream_);
    if (cudaGetLastError() != cudaSuccess) return fail("distance kernel launch");
    session_count_launches(1);
    if (cudaMemcpyAsync(hb + 16, db + 16, kOffOut - 16 + 4u * n, cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
      return fail("distance kernel");
    *gpu_us += static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count());
    return *reinterpret_cast<const int32_t*>(hb + 16) == 0;
  }

 private:
  bool fail(const char* what) {
    session_error("session %s: %s", what, cudaGetErrorString(cudaGetLastError()));
    return false;
  }

  size_t table_floats_ = 0;
  cudaStream_t stream_ = nullptr;
  void* d_block_ = nullptr;
  float* d_table_ = nullptr;
  void* h_block_ = nullptr;
};

// ---- host-side polling ------------------------------------------------------
inline void acquire_fence() { std::atomic_thread_fence(std::memory_order_acquire); }
inline void release_fence() { std::atomic_thread_fence(std::memory_order_release); }

// Idle limit of a session: a host that neither submits a buffer nor changes
// the session's state for this long is taken to be gone (ROVER_SESSION_IDLE_MS,
// default 60 s; 0 = no limit).
int64_t idle_limit_us() {
  const char* v = std::getenv("ROVER_SESSION_IDLE_MS");
  const long long ms = v ? std::atoll(v) : 60000;
  return ms <= 0 ? 0 : static_cast<int64_t>(ms) * 1000;
}

// Backs off while nothing is ready: spins first (the host fills buffers
// microseconds apart), then yields, then sleeps in short steps.
class Backoff {
 public:
  explicit Backoff(int64_t limit_us) : limit_us_(limit_us) { reset(); }
  void reset() {
    idle_polls_ = 0;
    since_ = std::chrono::steady_clock::now();
  }
  // Work arrived: adds the time spent waiting for it, and starts over.
  void woke(uint64_t* waited_us) {
    if (idle_polls_) *waited_us += idle_us();
    reset();
  }
  // false once the idle limit has passed
  bool wait(uint64_t* polls) {
    ++*polls;
    ++idle_polls_;
    if (idle_polls_ < 2000) return true;
    if (idle_polls_ < 4000) {
      std::this_thread::yield();
    } else {
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    return limit_us_ == 0 || static_cast<int64_t>(idle_us()) < limit_us_;
  }
  uint64_t idle_us() const {
    return static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - since_).count());
  }

 private:
  int64_t limit_us_;
  uint64_t idle_polls_ = 0;
  std::chrono::steady_clock::time_point since_;
};

// Host memory behind an rpcmem fd, at least `need` bytes.
template <class T>
T* map_fd(int fd, size_t need) {
  void* p = nullptr;
  size_t bytes = 0;
  if (fd < 0 || rover_rpcmem_lookup(fd, &p, &bytes) != 0 || !p || bytes < need) return nullptr;
  return static_cast<T*>(p);
}

// A ready buffer of a pass: where it is and where its ids start in the list.
struct Ready {
  int lane, index, first;
};

// ---- pure-PQ session ----------------------------------------------------------
//
// pure_pq_sqmd_process_buffer_payload (retrieval_sqmd_pure_pq.c:309-378)
// checks each buffer against the session's query generation and the LUT
// header (generations, m, ks, entry count, index uuid) and every work item's
// ids; a buffer that fails aborts the session (control state ABORT), as a
// DSP lane worker does (retrieval_async_dsp_search.c:2180-2240).
AEEResult serve_pure_pq(const SessionIndex& ix, PqControl* ctl, PqLutHeader* hdr, const float* lut, int lanes,
                        int cap) {
  const PqIndexView& v = ix.pq;
  const int entries = v.m * v.ks;
  GpuPass gpu;
  if (!gpu.init(static_cast<size_t>(entries))) return AEE_ENOMEMORY;
  // pure_pq_sqmd_control_init (retrieval_sqmd_pure_pq.c:280-307)
  std::memset(static_cast<void*>(ctl), 0, sizeof(*ctl));
  ctl->lane_count = lanes;
  for (int l = 0; l < kLanesMax; ++l) {
    ctl->lanes[l].dsp_active_buffer = -1;
    ctl->lanes[l].cpu_fill_buffer = 0;
  }
  ctl->control_state = kPqIdle;
  release_fence();
  ctl->control_state = kPqRunning;
  release_fence();

  Backoff idle(idle_limit_us());
  uint64_t compute_us = 0, wait_us = 0, polls = 0, aborts = 0;
  int table_gen = -1;     // query generation whose LUT is on the device
  AEEResult rc = AEE_SUCCESS;
  auto abort_session = [&](const char* why) {
    session_error("pure-PQ session aborted: %s", why);
    ++aborts;
    release_fence();
    ctl->control_state = kPqAbort;
    release_fence();
    rc = AEE_EFAILED;
  };
  for (;;) {
    acquire_fence();
    const int32_t state = ctl->control_state;
    if (state == kPqShutdown) break;
    if (state == kPqAbort) {
      if (rc == AEE_SUCCESS) session_error("pure-PQ session aborted by the host");
      rc = AEE_EFAILED;
      break;
    }
    Ready ready[kLanesMax * kBuffersPerLane];
    int nready = 0, nids = 0;
    for (int l = 0; l < lanes; ++l)
      for (int b = 0; b < kBuffersPerLane; ++b)
        if (ctl->lanes[l].buffers[b].state == kPqCpuReady) ready[nready++] = Ready{l, b, 0};
    if (nready == 0) {
      if (!idle.wait(&polls)) {
        abort_session("the host submitted nothing within the idle limit");
        break;
      }
      continue;
    }
    idle.woke(&wait_us);
    acquire_fence();
    const int32_t gen = ctl->query_gen;
    const char* bad = nullptr;
    for (int r = 0; r < nready && !bad; ++r) {
      const PqLaneBuffer& buf = ctl->lanes[ready[r].lane].buffers[ready[r].index];
      if (buf.query_gen != gen || buf.work_count < 0 || buf.work_count > cap) bad = "buffer generation or work count";
      else if (hdr->query_gen != gen || hdr->lut_gen != gen || hdr->m != v.m || hdr->ks != v.ks ||
               hdr->lut_count != entries || std::memcmp(hdr->index_uuid, ix.pq_uuid, 16) != 0)
        bad = "lookup-table header does not match the query or the index";
      ready[r].first = nids;
      for (int i = 0; i < buf.work_count && !bad; ++i) {
        const PqWork& w = buf.work[i];
        if (w.neighbor_id < 0 || w.neighbor_id >= v.n || w.source_id < 0 || w.source_id >= v.n)
          bad = "work item id out of range";
        else gpu.ids()[nids++] = w.neighbor_id;
      }
    }
    if (!bad && gen != table_gen) {
      if (!gpu.upload_table(lut, static_cast<size_t>(entries) * sizeof(float))) bad = "lookup-table upload";
      else table_gen = gen;
    }
    if (!bad && nids > 0 && !gpu.run(&v, nullptr, nids, &compute_us)) bad = "ADC kernel (non-finite distance or CUDA error)";
    if (bad) {
      abort_session(bad);
      break;
    }
    for (int r = 0; r < nready; ++r) {
      PqLane& lane = ctl->lanes[ready[r].lane];
      PqLaneBuffer& buf = lane.buffers[ready[r].index];
      lane.dsp_active_buffer = ready[r].index;
      for (int i = 0; i < buf.work_count; ++i) {
        buf.result[i].neighbor_id = buf.work[i].neighbor_id;
        buf.result[i].source_id = buf.work[i].source_id;
        buf.result[i].distance = gpu.out()[ready[r].first + i];
      }
      buf.result_count = buf.work_count;
      release_fence();
      buf.state = kPqDspDone;
      lane.dsp_active_buffer = -1;
    }
    release_fence();
  }
  acquire_fence();
  ctl->stats.dsp_compute_us += compute_us;
  ctl->stats.dsp_wait_cpu_us += wait_us;
  ctl->stats.dsp_wait_polls += polls;
  ctl->stats.abort_count += aborts;
  release_fence();
  return rc;
}

// ---- SQMD sessions ------------------------------------------------------------
//
// One service for both SQ entry points.  Per query (persistent == false,
// calculator_retrieval_expand_sqmd, retrieval_async_dsp_search.c:1584-1790):
// the query comes with the call and the session ends when the host sets the
// control state to DONE (or ABORT).  Persistent (calculator_retrieval_
// expand_sqmd_run, :1791-1990): the query is read from the control block's
// query slot whenever its generation changes, and the session ends at
// session state SHUTDOWN (or ABORT).  Buffers are checked as
// sqmd_process_lane_buffer_payload_with_cap does (retrieval_sqmd_common.c:
// 215-252): more items than the cap is TOO_MUCH_WORK, an id outside the index
// BAD_PARAM; the failure is recorded in the buffer (result_count = status,
// state DSP_ABORT) and the service stops serving, as the lane worker that
// met it exits (sqmd_dsp_worker_record_abort, :1018-1034).
AEEResult serve_sqmd(const SessionIndex& ix, SqControl* ctl, const float* call_query, int lanes, int cap,
                     bool persistent) {
  const SqIndexView& v = ix.sq;
  GpuPass gpu;
  if (!gpu.init(static_cast<size_t>(v.dim))) return AEE_ENOMEMORY;
  if (persistent) {
    ctl->session_state = kSessIdle;
    ctl->ctrl_state = kCtrlDone;
    ctl->query_slot.query_gen = 0;
  } else {
    ctl->ctrl_state = kCtrlPreparing;
  }
  ctl->lane_count = lanes;
  ctl->turn_id = 0;
  std::memset(const_cast<SqStats*>(&ctl->stats), 0, sizeof(ctl->stats));
  for (int l = 0; l < kLanesMax; ++l) {
    for (int b = 0; b < kBuffersPerLane; ++b) {
      SqLaneBuffer& buf = ctl->lanes[l].buf[b];
      buf.state = kSqEmpty;
      buf.turn_id = buf.work_count = buf.result_count = 0;
    }
    ctl->lanes[l].dsp_active_buf = -1;
    ctl->lanes[l].cpu_fill_buf = 0;
  }
  release_fence();
  uint64_t compute_us = 0, wait_us = 0, polls = 0, aborts = 0;
  AEEResult rc = AEE_SUCCESS;
  auto set_abort = [&]() {
    ++aborts;
    release_fence();
    if (persistent) ctl->session_state = kSessAbort;
    else ctl->ctrl_state = kCtrlAbort;
    release_fence();
    rc = AEE_EFAILED;
  };
  acquire_fence();
  if (ctl->startup_slot.cancel) {
    session_error("SQMD session cancelled by the host before it started");
    set_abort();
    return rc;
  }
  int table_gen = -1;
  bool aligned = false;   // the current query uses the ALIGNED_U8 contract
  if (!persistent) {
    if (!gpu.upload_table(call_query, static_cast<size_t>(v.dim) * sizeof(float))) return AEE_EFAILED;
    table_gen = 0;
  }
  release_fence();
  if (persistent) ctl->session_state = kSessRunning;
  else ctl->ctrl_state = kCtrlRunning;
  release_fence();

  Backoff idle(idle_limit_us());
  bool serving = true;
  for (;;) {
    acquire_fence();
    if (!ctl->startup_slot.acknowledged && ctl->startup_slot.cancel) {
      session_error("SQMD session cancelled by the host");
      set_abort();
      break;
    }
    if (persistent) {
      const int32_t ss = ctl->session_state;
      if (ss == kSessShutdown) break;
      if (ss == kSessAbort) { rc = AEE_EFAILED; break; }
      if (ctl->ctrl_state == kCtrlAbort) serving = false;   // the lane workers leave
    } else {
      const int32_t cs = ctl->ctrl_state;
      if (cs == kCtrlDone) break;
      if (cs == kCtrlAbort) { rc = AEE_EFAILED; break; }
    }
    Ready ready[kLanesMax * kBuffersPerLane];
    int nready = 0, nids = 0;
    if (serving)
      for (int l = 0; l < lanes; ++l)
        for (int b = 0; b < kBuffersPerLane; ++b)
          if (ctl->lanes[l].buf[b].state == kSqCpuReady) ready[nready++] = Ready{l, b, 0};
    if (nready == 0) {
      if (!idle.wait(&polls)) {
        session_error("SQMD session: the host changed nothing within the idle limit");
        set_abort();
        break;
      }
      continue;
    }
    idle.woke(&wait_us);
    acquire_fence();
    SqLaneBuffer* failed = nullptr;
    int32_t fail_status = 0;
    if (persistent && ctl->query_slot.query_gen != table_gen) {
      // the lane worker's query refresh (retrieval_async_dsp_search.c:1095-1127):
      // the legacy contract quantizes the FP32 query; the ALIGNED_U8
      // contract (split distance) hands over the host's u8 query, which
      // needs 4-bit L1 codes and the index's dimension
      const SqQuerySlot& qs = ctl->query_slot;
      const bool want_aligned = qs.contract_id == kContractAlignedU8;
      bool ok;
      if (want_aligned) {
        ok = qs.query_dim == v.dim && v.l1_bits == 4 && std::isfinite(v.l1_scale) && v.l1_scale > 0.0f &&
             gpu.upload_table(const_cast<const uint8_t*>(qs.query_u8), static_cast<size_t>(v.dim));
      } else {
        ok = qs.contract_id == kContractLegacy && v.l1_scale != 0.0f &&
             gpu.upload_table(const_cast<const float*>(qs.query), static_cast<size_t>(v.dim) * sizeof(float));
      }
      if (!ok) {
        failed = &ctl->lanes[ready[0].lane].buf[ready[0].index];
        fail_status = kSqStatusBadParam;
        session_error(want_aligned ? "SQMD session: the aligned-u8 query does not fit this index"
                      : qs.contract_id != kContractLegacy ? "SQMD session: unknown query contract"
                                                          : "SQMD session: the query cannot be quantized");
      } else {
        table_gen = qs.query_gen;
        aligned = want_aligned;
      }
    }
    for (int r = 0; r < nready && !failed; ++r) {
      SqLaneBuffer& buf = ctl->lanes[ready[r].lane].buf[ready[r].index];
      ready[r].first = nids;
      if (buf.work_count < 0) { failed = &buf; fail_status = kSqStatusBadParam; break; }
      if (buf.work_count > cap) { failed = &buf; fail_status = kSqStatusTooMuchWork; break; }
      for (int i = 0; i < buf.work_count; ++i) {
        const int32_t id = buf.work[i].neighbor_id;
        if (id < 0 || id >= v.n) { failed = &buf; fail_status = kSqStatusBadParam; break; }
        gpu.ids()[nids++] = id;
      }
    }
    if (!failed && nids > 0 && !gpu.run(nullptr, &v, nids, &compute_us, aligned)) {
      failed = &ctl->lanes[ready[0].lane].buf[ready[0].index];
      fail_status = kSqStatusBadParam;
    }
    if (failed) {
      // sqmd_dsp_worker_record_abort: the status in result_count, state DSP_ABORT
      failed->result_count = fail_status;
      release_fence();
      failed->state = kSqDspAbort;
      release_fence();
      ++aborts;
      rc = AEE_EFAILED;
      serving = false;
      continue;
    }
    for (int r = 0; r < nready; ++r) {
      SqLane& lane = ctl->lanes[ready[r].lane];
      SqLaneBuffer& buf = lane.buf[ready[r].index];
      lane.dsp_active_buf = ready[r].index;
      for (int i = 0; i < buf.work_count; ++i) {
        buf.result[i].neighbor_id = buf.work[i].neighbor_id;
        buf.result[i].source_id = buf.work[i].source_id;
        buf.result[i].coarse_dist = gpu.out()[ready[r].first + i];
      }
      buf.result_count = buf.work_count;
      release_fence();
      buf.state = kSqDspDone;
      lane.dsp_active_buf = -1;
    }
    release_fence();
  }
  acquire_fence();
  ctl->stats.dsp_compute_us += compute_us;
  ctl->stats.dsp_wait_cpu_us += wait_us;
  ctl->stats.dsp_wait_poll_count += polls;
  ctl->stats.abort_count += aborts;
  release_fence();
  return rc;
}

// Sessions run on the thread that calls them, which may not have made the
// library's device current: make it so for the session's lifetime.
class DeviceScope {
 public:
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != device) {
      if (cudaSetDevice(device) == cudaSuccess) restore_ = true;
    }
  }
  ~DeviceScope() {
    if (restore_) cudaSetDevice(prev_);
  }

 private:
  int prev_ = 0;
  bool restore_ = false;
};

}  // namespace
}  // namespace rover

using namespace rover;

// retrieval_async_dsp_search.c:2269-2479.  Argument checks as the
// reference's; the control block and the LUT buffer are rpcmem buffers
// named by their fds.  Blocks until the host sets SHUTDOWN (AEE_SUCCESS) or
// ABORT, or the session aborts itself (AEE_EFAILED).
extern "C" AEEResult calculator_retrieval_pure_pq_sqmd_run(remote_handle64 h, int32 fd_sqmd_ctrl, int32 fd_query_lut,
                                                           int32 lane_count, int32 work_items_cap) {
  (void)h;
  if (fd_sqmd_ctrl < 0 || fd_query_lut < 0 || lane_count <= 0 || lane_count > kLanesMax || work_items_cap <= 0 ||
      work_items_cap > kItemsMax) {
    session_error("pure-PQ session: bad fds, lane count or work cap");
    return AEE_EBADPARM;
  }
  SessionIndex ix;
  if (!session_acquire(kSessionPurePq, &ix)) return AEE_EBADPARM;
  DeviceScope device(ix.device);
  AEEResult rc = AEE_EFAILED;
  const size_t lut_bytes = sizeof(PqLutHeader) + static_cast<size_t>(ix.pq.m) * ix.pq.ks * sizeof(float);
  PqControl* ctl = map_fd<PqControl>(fd_sqmd_ctrl, sizeof(PqControl));
  PqLutHeader* hdr = map_fd<PqLutHeader>(fd_query_lut, lut_bytes);
  if (!ctl || !hdr) {
    session_error("pure-PQ session: an fd names no rpcmem buffer of the needed size");
  } else {
    const float* lut = reinterpret_cast<const float*>(reinterpret_cast<const uint8_t*>(hdr) + sizeof(PqLutHeader));
    rc = serve_pure_pq(ix, ctl, hdr, lut, lane_count, work_items_cap);
  }
  session_release(kSessionPurePq);
  return rc;
}

// retrieval_async_dsp_search.c:1584-1790: one query's SQMD expansions.
extern "C" AEEResult calculator_retrieval_expand_sqmd(remote_handle64 h, const float* query, int queryLen,
                                                      int32 query_dim, int32 fd_sqmd_ctrl, int32 lane_count,
                                                      int32 work_items_cap) {
  (void)h;
  if (!query || queryLen != query_dim || query_dim <= 0 || query_dim > kMaxDim || fd_sqmd_ctrl < 0 ||
      lane_count <= 0 || lane_count > kLanesMax || work_items_cap <= 0 || work_items_cap > kItemsMax) {
    session_error("SQMD session: bad query, fd, lane count or work cap");
    return AEE_EBADPARM;
  }
  SessionIndex ix;
  if (!session_acquire(kSessionSqmd, &ix)) return AEE_EFAILED;
  AEEResult rc = AEE_EFAILED;
  if (query_dim < ix.sq.dim || !(ix.sq.l1_scale != 0.0f)) {
    session_error("SQMD session: the query cannot be quantized for this index");
    rc = AEE_EBADPARM;
  } else if (SqControl* ctl = map_fd<SqControl>(fd_sqmd_ctrl, sizeof(SqControl))) {
    DeviceScope device(ix.device);
    rc = serve_sqmd(ix, ctl, query, lane_count, work_items_cap, false);
  } else {
    session_error("SQMD session: the fd names no rpcmem buffer of the needed size");
  }
  session_release(kSessionSqmd);
  return rc;
}

// retrieval_async_dsp_search.c:1791-1990: the persistent SQMD session.
extern "C" AEEResult calculator_retrieval_expand_sqmd_run(remote_handle64 h, int32 fd_sqmd_ctrl, int32 lane_count,
                                                          int32 work_items_cap) {
  (void)h;
  if (fd_sqmd_ctrl < 0 || lane_count <= 0 || lane_count > kLanesMax || work_items_cap <= 0 ||
      work_items_cap > kItemsMax) {
    session_error("SQMD session: bad fd, lane count or work cap");
    return AEE_EBADPARM;
  }
  SessionIndex ix;
  if (!session_acquire(kSessionSqmd, &ix)) return AEE_EFAILED;
  AEEResult rc = AEE_EFAILED;
  if (SqControl* ctl = map_fd<SqControl>(fd_sqmd_ctrl, sizeof(SqControl))) {
    DeviceScope device(ix.device);
    rc = serve_sqmd(ix, ctl, nullptr, lane_count, work_items_cap, true);
  } else {
    session_error("SQMD session: the fd names no rpcmem buffer of the needed size");
  }
  session_release(kSessionSqmd);
  return rc;
}

// ---- DB-pair search --------------------------------------------------------
//
// retrieval_async_dsp_search.c:1399-1581.  Two queries searched side by side;
// each expansion's neighbours go to the caller through the shared expansion
// buffer (DSP_DONE), the caller's correction thread writes their corrected
// distances back (CPU_DONE), and only then does the search take its next
// step.  Both searches live on the device (db_step_kernel); this loop moves
// each step's ids and distances between the expansion buffers and the
// device, one launch per round for every slot that is ready.
namespace {

struct DbDevice {
  cudaStream_t stream = nullptr;
  void* block = nullptr;
  DbIo* h_io = nullptr;
  bool ok = false;
  DbArgs args{};
  ~DbDevice() {
    if (stream) cudaStreamSynchronize(stream);
    if (block) cudaFree(block);
    if (h_io) cudaFreeHost(h_io);
    if (stream) cudaStreamDestroy(stream);
  }
  // One allocation: io, slots, queries, pools, frontiers, visited bitmaps, outputs.
  bool init(const SqIndexView& v, int pool_cap, int num_out) {
    const size_t n = static_cast<size_t>(v.n), vwords = (n + 31) / 32;
    auto up = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
    const size_t o_io = 0, o_slots = up(o_io + sizeof(DbIo)), o_q = up(o_slots + kDbSlots * sizeof(DbSlot)),
                 o_pool = up(o_q + kDbSlots * v.dim * 4ull), o_front = up(o_pool + kDbSlots * pool_cap * 8ull),
                 o_vis = up(o_front + kDbSlots * n * 8), o_ids = up(o_vis + kDbSlots * vwords * 4),
                 o_d = up(o_ids + kDbSlots * num_out * 4ull), total = up(o_d + kDbSlots * num_out * 4ull);
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&block, total) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&h_io), sizeof(DbIo), cudaHostAllocDefault) != cudaSuccess) {
      session_error("DB-pair set-up: %s", cudaGetErrorString(cudaGetLastError()));
      return false;
    }
    uint8_t* b = static_cast<uint8_t*>(block);
    args.ix = v;
    args.io = reinterpret_cast<DbIo*>(b + o_io);
    args.slots = reinterpret_cast<DbSlot*>(b + o_slots);
    args.queries = reinterpret_cast<const float*>(b + o_q);
    args.pools = reinterpret_cast<uint64_t*>(b + o_pool);
    args.fronts = reinterpret_cast<uint64_t*>(b + o_front);
    args.visited = reinterpret_cast<uint32_t*>(b + o_vis);
    args.out_ids = reinterpret_cast<int32_t*>(b + o_ids);
    args.out_dists = reinterpret_cast<float*>(b + o_d);
    args.pool_cap = pool_cap;
    args.num_out = num_out;
    args.frontier_cap = v.n;     // every id enters the frontier at most once
    std::memset(h_io, 0, sizeof(DbIo));
    return ok = true;
  }
  bool upload_queries(const float* qa, const float* qb) {
    float* q = const_cast<float*>(args.queries);
    const size_t bytes = static_cast<size_t>(args.ix.dim) * 4;
    return cudaMemcpyAsync(q, qa, bytes, cudaMemcpyHostToDevice, stream) == cudaSuccess &&
           cudaMemcpyAsync(q + args.ix.dim, qb, bytes, cudaMemcpyHostToDevice, stream) == cudaSuccess;
  }
  // h_io -> device, one step, device -> h_io
  bool launch() {
    if (cudaMemcpyAsync(args.io, h_io, sizeof(DbIo), cudaMemcpyHostToDevice, stream) != cudaSuccess) return false;
    launch_db_step(args, stream);
    if (cudaGetLastError() != cudaSuccess) return false;
    session_count_launches(1);
    return cudaMemcpyAsync(h_io, args.io, sizeof(DbIo), cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
           cudaStreamSynchronize(stream) == cudaSuccess;
  }
};

}  // namespace

extern "C" AEEResult calculator_retrieval_search_db(remote_handle64 h, const float* query_a, int query_aLen,
                                                    const float* query_b, int query_bLen, int32 fd_expansion_buf,
                                                    int32 entry_points, int32 expand_count, int32 pool_size,
                                                    int32 num_out, int* candidate_ids_a, int candidate_ids_aLen,
                                                    float* candidate_dists_a, int candidate_dists_aLen,
                                                    int32* actual_count_a, int* candidate_ids_b, int candidate_ids_bLen,
                                                    float* candidate_dists_b, int candidate_dists_bLen,
                                                    int32* actual_count_b) {
  (void)h;
  if (!actual_count_a || !actual_count_b) return AEE_EBADPARM;
  *actual_count_a = 0;
  *actual_count_b = 0;
  DbShared* shared = map_fd<DbShared>(fd_expansion_buf, sizeof(DbShared));
  if (!shared) {
    session_error("DB-pair search: the fd names no rpcmem buffer of the needed size");
    return AEE_EFAILED;
  }
  SessionIndex ix;
  if (!session_acquire(kSessionDb, &ix)) return AEE_EFAILED;
  struct Release { ~Release() { session_release(kSessionDb); } } release;
  const SqIndexView& v = ix.sq;
  if (!v.graph) {
    session_error("DB-pair search: the loaded L1 index has no graph");
    return AEE_EFAILED;
  }
  if (candidate_ids_aLen < num_out || candidate_dists_aLen < num_out || candidate_ids_bLen < num_out ||
      candidate_dists_bLen < num_out)
    return AEE_EBADPARM;
  // db_search_state_init's refusals (:1213-1224, quantization at :1270)
  const int expand_limit = std::min(expand_count, v.degree);
  if (!query_a || !query_b || query_aLen < v.dim || query_bLen < v.dim || entry_points <= 0 || pool_size <= 0 ||
      num_out <= 0 || expand_limit <= 0 || !(v.l1_scale != 0.0f)) {
    session_error("DB-pair search: the search state cannot be set up for these arguments");
    return AEE_ENOMEMORY;
  }
  DeviceScope device(ix.device);
  const int cap = std::min(pool_size, 2000);   // DSP_SEARCH_MAX_POOL
  DbDevice dev;
  if (!dev.init(v, cap, num_out) || !dev.upload_queries(query_a, query_b)) return AEE_ENOMEMORY;
  dev.args.entry_points = entry_points;
  dev.args.expand_limit = std::min(expand_limit, kItemsMax);
  dev.args.graph_entry = ix.sq_graph_entry;   // as dsp_search_select_entry_id reads it
  DbIo& io = *dev.h_io;
  io.op[0] = io.op[1] = kDbInit;
  if (!dev.launch() || io.status[0] != kStatusOk || io.status[1] != kStatusOk) {
    session_error("DB-pair search: entry seeding failed");
    return AEE_ENOMEMORY;
  }
  for (int i = 0; i < 2; ++i) {
    shared->buf[i].state = kDbEmpty;
    shared->buf[i].finished = 0;
    shared->buf[i].count = 0;
  }
  shared->stats.dsp_wait_cpu_done_us = shared->stats.dsp_invalidate_us = shared->stats.dsp_wait_poll_count = 0;
  release_fence();
  bool fin[2] = {false, false};
  Backoff idle(idle_limit_us());
  uint64_t wait_us = 0, polls = 0;
  while (!fin[0] || !fin[1]) {
    acquire_fence();
    bool any = false;
    for (int i = 0; i < 2; ++i) {
      io.op[i] = kDbNone;
      if (fin[i]) continue;
      DbExpansion& b = shared->buf[i];
      const int32_t state = b.state;
      if (state == kDbCpuDone) {
        acquire_fence();
        if (b.count < 0 || b.count > kItemsMax) return AEE_ENOMEMORY;   // db_search_apply_corrections refuses
        for (int j = 0; j < b.count; ++j) io.corr[i][j] = b.corrected_dists[j];
        io.op[i] = kDbStep;
      } else if (state == kDbEmpty) {
        io.op[i] = kDbStep;
      }
      any |= io.op[i] != kDbNone;
    }
    if (!any) {
      if (!idle.wait(&polls)) {
        session_error("DB-pair search: the caller returned no corrections within the idle limit");
        return AEE_EFAILED;
      }
      continue;
    }
    idle.woke(&wait_us);
    if (!dev.launch()) {
      session_error("DB-pair search: %s", cudaGetErrorString(cudaGetLastError()));
      return AEE_EFAILED;
    }
    for (int i = 0; i < 2; ++i) {
      if (io.op[i] != kDbStep) continue;
      if (io.status[i] != kStatusOk) {
        session_error("DB-pair search: step failed with status %d", io.status[i]);
        return AEE_ENOMEMORY;
      }
      DbExpansion& b = shared->buf[i];
      if (io.finished[i]) {
        fin[i] = true;
        b.finished = 1;
        b.count = 0;
      } else {
        for (int j = 0; j < io.count[i]; ++j) {
          b.neighbor_ids[j] = io.ids[i][j];
          b.coarse_dists[j] = io.coarse[i][j];
        }
        b.count = io.count[i];
      }
      release_fence();
      b.state = kDbDspDone;
    }
  }
  io.op[0] = io.op[1] = kDbFinish;
  if (!dev.launch()) return AEE_EFAILED;
  const int na = io.out_count[0], nb = io.out_count[1];
  const size_t bytes_a = static_cast<size_t>(na) * 4, bytes_b = static_cast<size_t>(nb) * 4;
  const bool copied =
      cudaMemcpyAsync(candidate_ids_a, dev.args.out_ids, bytes_a, cudaMemcpyDeviceToHost, dev.stream) == cudaSuccess &&
      cudaMemcpyAsync(candidate_dists_a, dev.args.out_dists, bytes_a, cudaMemcpyDeviceToHost, dev.stream) == cudaSuccess &&
      cudaMemcpyAsync(candidate_ids_b, dev.args.out_ids + num_out, bytes_b, cudaMemcpyDeviceToHost, dev.stream) == cudaSuccess &&
      cudaMemcpyAsync(candidate_dists_b, dev.args.out_dists + num_out, bytes_b, cudaMemcpyDeviceToHost, dev.stream) == cudaSuccess &&
      cudaStreamSynchronize(dev.stream) == cudaSuccess;
  if (!copied) return AEE_EFAILED;
  *actual_count_a = na;
  *actual_count_b = nb;
  shared->stats.dsp_wait_cpu_done_us = wait_us;
  shared->stats.dsp_wait_poll_count = polls;
  release_fence();
  return AEE_SUCCESS;
}
