// calculator.cu -- libcalculator.so: Rover's accelerator C-ABI on a B200.
//
// The reference serves these entry points from a Hexagon DSP skeleton whose
// state is module-global (src/dsp_demo/retrieval_async_dsp_search.c:44-76:
// one loaded index per process).  This library keeps the same model: one
// process-wide device state guarded by a mutex, shared by every session
// handle.  Index buffers are uploaded to HBM once at load time; searches run
// as the kernels in pq_search.cu / sq_search.cu / distance.cu.

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/calculator.h"
#include "../../include/rover_b200.h"
#include "kernels.h"
#include "rpcmem_compat.h"
#include "session_bridge.h"

using namespace rover;

namespace {

thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

#define CK(expr)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (expr);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return AEE_EFAILED;                                                            \
    }                                                                                \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b ? b : 16);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// The entry seeds of one (entry_points, seed) request: the distinct ids in
// draw order plus a bitmap of them.  Queries share them.
struct SeedSet {
  bool valid = false;
  int32_t entries = 0;
  uint32_t seed = 0;
  int32_t count = 0, dups = 0;
  DevBuf ids, bits;
  bool recon_ready = false;        // PQ reconstructions for ranking (gated search, traces)
  DevBuf recon, recon_norms;
  bool drows_ready = false;        // decoded rows for the verified exact seed pool
  DevBuf drows, drow_norms;
  // TF32-rounded copies of recon / drows named by TMA descriptors, for the
  // tensor-core seed ranking (valid == 0: the mma.sync ranking is used)
  DevBuf recon_tc, drows_tc;
  TcSeedMap recon_map{}, drows_map{};
  float drow_norm_max = 0.0f;      // largest of drow_norms (+inf if one is not finite)
  void release() {
    ids.release(); bits.release(); recon.release(); recon_norms.release(); drows.release(); drow_norms.release();
    recon_tc.release(); drows_tc.release();
    recon_map.valid = 0;
    drows_map.valid = 0;
    valid = false;
    recon_ready = false;
    drows_ready = false;
  }
};

struct PqDevice {
  DevBuf graph, codes, codebook, residual, qparams;
  DevBuf e4_qparams, e4_blocks;   // ERROR4 artifact (calculator_rover_error4_load)
  DevBuf decoded;                 // [n][dim] FP32 reconstructions, built on first use
  bool decoded_ready = false;
  SeedSet seeds;
  PqIndexView view{};
  int32_t graph_entry = -1;
  bool loaded = false;
  bool has_graph = false;
  uint64_t epoch = 0;             // bumped whenever the device copy is released (plans check it)
  void release() {
    graph.release(); codes.release(); codebook.release(); residual.release(); qparams.release();
    decoded.release(); seeds.release(); e4_qparams.release(); e4_blocks.release();
    view.e4 = Error4View{};
    decoded_ready = false;
    loaded = false;
    has_graph = false;
    ++epoch;
  }
};

struct SqDevice {
  DevBuf graph, l1, residual, qparams;
  DevBuf e4_qparams, e4_blocks;   // ERROR4 artifact (calculator_rover_error4_load)
  DevBuf split_bias;              // SQ4 split-distance bias (calculator_rover_sq_split_load)
  DevBuf entry_ids;               // entry ids of the last request (sq_entries)
  bool entries_valid = false, entries_sqmd = false;
  int32_t entries_target = 0, entry_count = 0;
  uint32_t entries_seed = 0;
  SqIndexView view{};
  int32_t graph_entry = -1;
  bool loaded = false;
  void release() {
    graph.release(); l1.release(); residual.release(); qparams.release();
    e4_qparams.release(); e4_blocks.release(); split_bias.release(); entry_ids.release();
    entries_valid = false;
    view.e4 = Error4View{};
    view.split_bias = nullptr;
    loaded = false;
  }
};

// Page-locked host memory that only grows (cudaHostAlloc).
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    const size_t want = std::max<size_t>(std::max<size_t>(b, 2 * bytes), 64);
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// A device-to-host copy the status fetch of a search enqueues with its own
// (fetch_status): the results of a host-buffer call land in page-locked
// staging in the same wait as the status.
struct EarlyCopy {
  void* dst;
  const void* src;
  size_t bytes;
};

struct State {
  std::mutex mu;
  bool init = false;
  int session_live[kSessionKinds] = {};   // sessions / DB-pair calls (SessionKind) holding an index
  uint8_t pq_uuid[16] = {};       // index uuid of the pure-PQ DMA index (session LUT checks)
  int device = -1;                // the device current at the first call: index copies, stream, scratch
  int sms = 0;
  cudaStream_t stream = nullptr;
  int32_t l1_bits = 4;           // calculator_rover_configure
  PqDevice pq;                    // extension PQ index / pure-PQ DMA index
  SqDevice sq;                    // extension SQ index
  SqDevice legacy;                // calculator_retrieval_load(_dma) index
  bool legacy_dma = false;
  // scratch
  DevBuf visited, heaps, counter, status, stats, luts, seed_dists, seed_rank;
  DevBuf seed_top, seed_top_next;  // per query: top-M seed ranks (pq_seed_topm_kernel)
  DevBuf tc_err;                   // set by the tensor-core seed ranking if a bounded wait ran out
  DevBuf gate_buf;                // BF16 transposed weights + FP32 biases of the loaded gate
  GateParams gate{};              // enabled == 0: no gate loaded
  DevBuf trace_rows, trace_count; // calculator_rover_pq_trace
  GateTraceRow* trace_dev = nullptr;
  unsigned long long* trace_count_dev = nullptr;
  int64_t trace_cap = 0;
  uint32_t visited_mask = 0;
  size_t visited_slots = 0;
  uint32_t gen_next = 1;
  DevBuf in_queries, in_pool, in_topk, in_ids, in_offsets;
  DevBuf out_ids, out_dists, out_counts, pool_ids, pool_dists, pool_counts;
  std::vector<int32_t> h_status;
  PinnedBuf status_pin, stage;    // page-locked status and result staging (fetch_status, pq_search_host)
  // Queries uploaded in pieces on copy_stream (pq_search_host): rows
  // [k arrival_rows, (k + 1) arrival_rows) are on the device once
  // arrival_ev[k] completes.  arrival_pieces == 0: nothing in flight.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t arrival_ev[4] = {};
  int arrival_rows = 0, arrival_pieces = 0;
  std::vector<EarlyCopy> early;   // result copies to enqueue with each status fetch of the current call
  bool early_done = false;        // a status fetch of the current call enqueued them
};

State& st() {
  static State s;
  return s;
}

int open_count = 0;
std::atomic<unsigned long long> g_launches{0};  // kernels this library launched

// Optional per-kernel event timing (calculator_rover_kernel_timing).
struct KernelTimer {
  std::mutex mu;
  bool on = false;
  struct Pending { int kind; cudaEvent_t start, stop; };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> spare;
  int64_t launches[ROVER_KERNEL_KINDS] = {};
  double ms[ROVER_KERNEL_KINDS] = {};
  cudaEvent_t take() {
    if (!spare.empty()) {
      cudaEvent_t e = spare.back();
      spare.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
  }
};

KernelTimer& timer() {
  static KernelTimer t;
  return t;
}

// Brackets one launch with events when timing is on.
class TimedLaunch {
 public:
  TimedLaunch(int kind, cudaStream_t s, bool enable = true) : kind_(kind), s_(s) {
    if (!enable) return;
    KernelTimer& t = timer();
    std::lock_guard<std::mutex> g(t.mu);
    if (!t.on) return;
    start_ = t.take();
    stop_ = t.take();
    if (start_ && stop_) cudaEventRecord(start_, s_);
  }
  ~TimedLaunch() {
    if (!start_ || !stop_) return;
    cudaEventRecord(stop_, s_);
    KernelTimer& t = timer();
    std::lock_guard<std::mutex> g(t.mu);
    t.pending.push_back({kind_, start_, stop_});
  }
  TimedLaunch(const TimedLaunch&) = delete;
  TimedLaunch& operator=(const TimedLaunch&) = delete;

 private:
  int kind_;
  cudaStream_t s_;
  cudaEvent_t start_ = nullptr, stop_ = nullptr;
};

// Reads the events of finished launches (call after the stream synchronized).
// Reads the events of finished launches; launches still in flight stay
// pending for a later call.
void collect_timings() {
  KernelTimer& t = timer();
  std::lock_guard<std::mutex> g(t.mu);
  std::vector<KernelTimer::Pending> running;
  for (const auto& p : t.pending) {
    if (cudaEventQuery(p.stop) == cudaErrorNotReady) {
      running.push_back(p);
      continue;
    }
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
      t.launches[p.kind] += 1;
      t.ms[p.kind] += ms;
    }
    cudaGetLastError();
    t.spare.push_back(p.start);
    t.spare.push_back(p.stop);
  }
  t.pending.swap(running);
}

AEEResult ensure_init(State& s) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (s.init) {
    // the index copies, the stream and the scratch live on s.device: a call
    // made with another device current would hand that device's kernels
    // pointers it cannot use, so it is refused before anything is launched
    if (dev != s.device) {
      set_error("device %d is current, but this library's state lives on device %d", dev, s.device);
      return AEE_EFAILED;
    }
    return AEE_SUCCESS;
  }
  CK(cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&s.copy_stream, cudaStreamNonBlocking));
  for (cudaEvent_t& e : s.arrival_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  s.device = dev;
  s.init = true;
  return AEE_SUCCESS;
}

// A live lane-protocol session reads the index it was started on: loading,
// replacing or unloading that index is refused until the session returns.
bool session_busy(const State& s, SessionKind k) {
  if (k == kSessionSqmd && s.session_live[kSessionDb]) k = kSessionDb;
  if (!s.session_live[k]) return false;
  set_error("a %s is running on the loaded index",
            k == kSessionPurePq ? "pure-PQ session" : k == kSessionSqmd ? "SQMD session" : "DB-pair search");
  return true;
}

template <class T>
AEEResult upload(DevBuf& b, const T* src, size_t count, cudaStream_t s) {
  CK(b.ensure(count * sizeof(T)));
  if (count) CK(cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
  return AEE_SUCCESS;
}

// The per-query statuses of a search, after everything enqueued on stream:
// one page-locked copy (with the call's early result copies) and one wait.
AEEResult fetch_status(State& s, const int32_t* d_status, int nq, cudaStream_t stream) {
  for (const EarlyCopy& c : s.early)
    CK(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, stream));
  s.early_done = !s.early.empty();
  CK(s.status_pin.ensure(static_cast<size_t>(nq) * sizeof(int32_t)));
  CK(cudaMemcpyAsync(s.status_pin.p, d_status, static_cast<size_t>(nq) * sizeof(int32_t), cudaMemcpyDeviceToHost,
                     stream));
  CK(cudaStreamSynchronize(stream));
  s.h_status.assign(s.status_pin.as<int32_t>(), s.status_pin.as<int32_t>() + nq);
  return AEE_SUCCESS;
}

// Makes stream wait until query rows [0, q_end) of a piecewise upload have
// arrived (no-op without one).
AEEResult await_rows(State& s, cudaStream_t stream, int q_end) {
  if (!s.arrival_pieces || q_end <= 0) return AEE_SUCCESS;
  const int k = std::min(s.arrival_pieces - 1, (q_end - 1) / s.arrival_rows);
  CK(cudaStreamWaitEvent(stream, s.arrival_ev[k], 0));
  return AEE_SUCCESS;
}

AEEResult seed_rank(State& s, const float* queries, int q0, int q1, int dim, const TcSeedMap& map,
                    const DevBuf& rows, const DevBuf& norms, int n_seeds, float* out, int stride, cudaStream_t st);

// TF32 ranks of queries [q0, q1) against the seed rows, then each query's
// top_m smallest (pq_seed_topm_kernel), into rows (q - q0) of rank / top /
// next.  With a piecewise query upload, each piece is ranked as soon as it
// has arrived, so the upload of the next overlaps the work.
AEEResult ranked_seeds(State& s, cudaStream_t stream, const float* queries, int q0, int q1, int dim,
                       const TcSeedMap& map, const DevBuf& rows, const DevBuf& norms, int n_seeds, float* rank,
                       int stride, int top_m, uint64_t* top, float* next) {
  for (int p0 = q0; p0 < q1;) {
    const int p1 = s.arrival_pieces ? std::min(q1, (p0 / s.arrival_rows + 1) * s.arrival_rows) : q1;
    if (await_rows(s, stream, p1) != AEE_SUCCESS) return AEE_EFAILED;
    const size_t off = static_cast<size_t>(p0 - q0);
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEED_RANK, stream);
      if (seed_rank(s, queries, p0, p1, dim, map, rows, norms, n_seeds, rank + off * stride, stride, stream) !=
          AEE_SUCCESS)
        return AEE_EFAILED;
    }
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEED_TOPM, stream);
      launch_pq_seed_topm(rank + off * stride, stride, n_seeds, p1 - p0, top_m, top + off * top_m, next + off,
                          stream);
    }
    CK(cudaGetLastError());
    g_launches += 2;
    p0 = p1;
  }
  return AEE_SUCCESS;
}

// The results of a host-buffer search: they travel within the search's own
// status fetch (one wait, no second round trip), straight into caller
// buffers that are page-locked, through page-locked staging into the
// others.  add() the (caller, device) pairs, arm() before the search,
// finish() after it succeeded.
class ResultStage {
 public:
  explicit ResultStage(State& s) : s_(s) {}
  ~ResultStage() {
    s_.early.clear();
    s_.early_done = false;
  }
  ResultStage(const ResultStage&) = delete;
  ResultStage& operator=(const ResultStage&) = delete;
  // A caller buffer in page-locked memory receives its copy directly.
  void add(void* user, const void* dev, size_t bytes) {
    if (!user || !dev || !bytes) return;
    cudaPointerAttributes at{};
    const bool pinned = cudaPointerGetAttributes(&at, user) == cudaSuccess && at.type == cudaMemoryTypeHost;
    if (!pinned) cudaGetLastError();
    parts_.push_back({user, dev, pinned ? 0 : total_, bytes, pinned});
    if (!pinned) total_ += (bytes + 255) & ~static_cast<size_t>(255);
  }
  AEEResult arm() {
    s_.early.clear();
    s_.early_done = false;
    if (total_ && s_.stage.ensure(total_) != cudaSuccess) return AEE_ENOMEMORY;
    for (const Part& x : parts_)
      s_.early.push_back({x.pinned ? x.user : s_.stage.as<uint8_t>() + x.off, x.dev, x.bytes});
    return AEE_SUCCESS;
  }
  AEEResult finish(cudaStream_t stream) {
    if (!parts_.empty() && !s_.early_done) {
      // a search path that returned without a status fetch: copy directly
      for (const Part& x : parts_) CK(cudaMemcpyAsync(x.user, x.dev, x.bytes, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      return AEE_SUCCESS;
    }
    for (const Part& x : parts_)
      if (!x.pinned) std::memcpy(x.user, s_.stage.as<uint8_t>() + x.off, x.bytes);
    return AEE_SUCCESS;
  }

 private:
  struct Part {
    void* user;
    const void* dev;
    size_t off, bytes;
    bool pinned;
  };
  State& s_;
  std::vector<Part> parts_;
  size_t total_ = 0;
};

uint32_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return static_cast<uint32_t>(p > 0x80000000ull ? 0x80000000ull : p);
}

// Reserve `entries` visited-table entries for each of `slots` warp slots and
// a generation range of `queries` queries.
AEEResult reserve_visited(State& s, size_t slots, uint32_t entries, uint32_t queries, uint32_t* gen_base) {
  const size_t need = slots * static_cast<size_t>(entries) * 8u;
  const bool regrow = need > s.visited.bytes || entries != s.visited_mask + 1u || slots > s.visited_slots;
  if (regrow || static_cast<uint64_t>(s.gen_next) + queries >= 0xffffffffull) {
    if (need > s.visited.bytes) CK(s.visited.ensure(need));
    CK(cudaMemsetAsync(s.visited.p, 0, need, s.stream));
    s.visited_mask = entries - 1u;
    s.visited_slots = slots;
    s.gen_next = 1;
  }
  *gen_base = s.gen_next;
  s.gen_next += queries;
  return AEE_SUCCESS;
}

int resident_blocks(const void* kernel, int threads, size_t smem, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * sms;
}

// Raises a kernel's dynamic shared-memory limit to at least `bytes` and never
// lowers it: plans set the limit once when they are made, and their launches
// (possibly replayed from a CUDA graph) must not find it lowered by a later
// search with smaller slices.  Callers hold the state lock.
AEEResult allow_smem(const void* fn, size_t bytes) {
  static std::vector<std::pair<const void*, size_t>> limits;
  for (auto& e : limits) {
    if (e.first != fn) continue;
    if (e.second >= bytes) return AEE_SUCCESS;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    e.second = bytes;
    return AEE_SUCCESS;
  }
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
  limits.emplace_back(fn, bytes);
  return AEE_SUCCESS;
}

// The largest seed filter (in bits: 64 Ki down to 8 Ki) that leaves the
// kernel's resident CTAs per SM unchanged next to warp slices of `slices`
// bytes per CTA; 0 when even the smallest would cost a CTA.
int seed_filter_bits(const void* kernel, int threads, size_t slices) {
  if (allow_smem(kernel, std::min<size_t>(slices + 8192, 227 * 1024)) != AEE_SUCCESS) return 0;
  int base = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&base, kernel, threads, slices) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int bits = 65536; bits >= 8192; bits >>= 1) {
    const size_t total = slices + bits / 8;
    if (total > 227 * 1024) continue;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, total) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (occ >= base) return bits;
  }
  return 0;
}

bool valid_params(const RoverSearchParams* p) {
  return p && p->size >= static_cast<int32_t>(offsetof(RoverSearchParams, reserved)) && p->entry_points > 0 &&
         p->expand_count > 0 && p->refine_budget >= 0 && p->refine_budget <= 2000 &&
         p->layout >= ROVER_LAYOUT_AUTO && p->layout <= ROVER_LAYOUT_DECODED;
}

// Entry seeds as pure_pq_make_seed_ids draws them
// (src/dsp_demo/retrieval_rpc_demo_pure_pq.c:192-208): the graph entry first
// (when valid), then id = (seed * n) >> 32 after each LCG step; a draw that
// repeats an earlier id is skipped as the search's visited check skips it
// (retrieval_sqmd_pure_pq.c:846-850).
AEEResult ensure_seeds(State& s, PqDevice& pq, int32_t entry_points, uint32_t seed) {
  const int32_t n = pq.view.n;
  const int32_t entries = std::min(entry_points, n);
  SeedSet& ss = pq.seeds;
  if (ss.valid && ss.entries == entries && ss.seed == seed) return AEE_SUCCESS;
  ss.valid = false;
  std::vector<uint32_t> bits((static_cast<size_t>(n) + 31) / 32, 0u);
  std::vector<int32_t> ids;
  ids.reserve(entries);
  int32_t dups = 0;
  uint32_t lcg = seed;
  for (int32_t i = 0; i < entries; ++i) {
    int32_t id;
    if (i == 0 && pq.graph_entry >= 0 && pq.graph_entry < n) {
      id = pq.graph_entry;
    } else {
      lcg = lcg * 1103515245u + 12345u;
      id = static_cast<int32_t>((static_cast<uint64_t>(lcg) * static_cast<uint64_t>(n)) >> 32);
    }
    uint32_t& w = bits[static_cast<uint32_t>(id) >> 5];
    const uint32_t bit = 1u << (static_cast<uint32_t>(id) & 31u);
    if (w & bit) {
      ++dups;
    } else {
      w |= bit;
      ids.push_back(id);
    }
  }
  if (upload(ss.ids, ids.data(), ids.size(), s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  if (upload(ss.bits, bits.data(), bits.size(), s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(cudaStreamSynchronize(s.stream));
  ss.entries = entries;
  ss.seed = seed;
  ss.count = static_cast<int32_t>(ids.size());
  ss.dups = dups;
  ss.valid = true;
  ss.recon_ready = false;
  ss.drows_ready = false;
  return AEE_SUCCESS;
}

// PQ reconstructions of the current seed set (for the tensor-core ranking).
// The tensor-core seed ranking runs where its descriptor could be made
// (dim 32..128 in steps of 32) unless ROVER_SEED_RANK=mma asks for the
// mma.sync kernel.
bool tc_rank_wanted() {
  static const bool want = [] {
    const char* v = std::getenv("ROVER_SEED_RANK");
    return !(v && std::strcmp(v, "mma") == 0);
  }();
  return want;
}

// A TF32-rounded copy of [count][dim] seed rows and its TMA descriptor.
AEEResult make_tc_rows(State& s, const DevBuf& rows, int count, int dim, DevBuf& copy, TcSeedMap& map) {
  map.valid = 0;
  if (!tc_rank_wanted() || !seed_rank_tc_supported(dim) || count <= 0) return AEE_SUCCESS;
  CK(copy.ensure(static_cast<size_t>(count) * dim * sizeof(float)));
  launch_tf32_round(rows.as<float>(), copy.as<float>(), static_cast<size_t>(count) * dim, s.stream);
  CK(cudaGetLastError());
  ++g_launches;
  if (!s.tc_err.p) {
    CK(s.tc_err.ensure(sizeof(int)));
    CK(cudaMemsetAsync(s.tc_err.p, 0, sizeof(int), s.stream));
  }
  tc_seed_map_encode(&map, copy.as<float>(), count, dim);   // invalid map: the mma.sync ranking
  return AEE_SUCCESS;
}

// Seed ranks of queries [q0, q1) into out: tensor cores when the rows have
// a descriptor, else mma.sync.
AEEResult seed_rank(State& s, const float* queries, int q0, int q1, int dim, const TcSeedMap& map,
                    const DevBuf& rows, const DevBuf& norms, int n_seeds, float* out, int stride, cudaStream_t st) {
  if (map.valid && launch_pq_seed_rank_tc(map, queries, q0, q1, dim, norms.as<float>(), n_seeds, out, stride,
                                          s.tc_err.as<int>(), s.sms, st))
    return AEE_SUCCESS;
  launch_pq_seed_rank(queries, q0, q1, dim, rows.as<float>(), norms.as<float>(), n_seeds, out, st, stride);
  CK(cudaGetLastError());
  return AEE_SUCCESS;
}

// After a search: fails the call if the tensor-core ranking gave up waiting.
AEEResult check_tc_err(State& s) {
  if (!s.tc_err.p) return AEE_SUCCESS;
  int e = 0;
  CK(cudaMemcpy(&e, s.tc_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(s.tc_err.p, 0, sizeof(int)));
    set_error("the tensor-core seed ranking gave up waiting on its pipeline; the search was not completed");
    return AEE_EFAILED;
  }
  return AEE_SUCCESS;
}

AEEResult ensure_seed_recon(State& s, PqDevice& pq) {
  SeedSet& ss = pq.seeds;
  if (ss.recon_ready) return AEE_SUCCESS;
  CK(ss.recon.ensure(static_cast<size_t>(ss.count) * pq.view.dim * sizeof(float)));
  CK(ss.recon_norms.ensure(static_cast<size_t>(ss.count) * sizeof(float)));
  launch_pq_seed_recon(pq.view, ss.ids.as<int32_t>(), ss.count, ss.recon.as<float>(), ss.recon_norms.as<float>(),
                       s.stream);
  CK(cudaGetLastError());
  ++g_launches;
  if (make_tc_rows(s, ss.recon, ss.count, pq.view.dim, ss.recon_tc, ss.recon_map) != AEE_SUCCESS) return AEE_EFAILED;
  CK(cudaStreamSynchronize(s.stream));
  ss.recon_ready = true;
  return AEE_SUCCESS;
}

// The current seed set's decoded rows and their norms (the TF32 ranking of
// the verified exact seed pool).  Needs the decoded rows.
AEEResult ensure_seed_drows(State& s, PqDevice& pq) {
  SeedSet& ss = pq.seeds;
  if (ss.drows_ready) return AEE_SUCCESS;
  CK(ss.drows.ensure(static_cast<size_t>(ss.count) * pq.view.dim * sizeof(float)));
  CK(ss.drow_norms.ensure(static_cast<size_t>(ss.count) * sizeof(float)));
  launch_pq_seed_gather(pq.decoded.as<float>(), pq.view.dim, ss.ids.as<int32_t>(), ss.count, ss.drows.as<float>(),
                        ss.drow_norms.as<float>(), s.stream);
  CK(cudaGetLastError());
  ++g_launches;
  if (make_tc_rows(s, ss.drows, ss.count, pq.view.dim, ss.drows_tc, ss.drows_map) != AEE_SUCCESS) return AEE_EFAILED;
  std::vector<float> norms(ss.count);
  CK(cudaMemcpyAsync(norms.data(), ss.drow_norms.p, norms.size() * sizeof(float), cudaMemcpyDeviceToHost, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  float mx = 0.0f;
  for (float v : norms) mx = std::isfinite(v) ? std::max(mx, v) : INFINITY;
  ss.drow_norm_max = mx;
  ss.drows_ready = true;
  return AEE_SUCCESS;
}

// Builds the decoded rows once per loaded index.  *ok = false when they do
// not fit (the caller then uses the packed layout).
AEEResult ensure_decoded(State& s, PqDevice& pq, bool* ok) {
  *ok = false;
  if (pq.decoded_ready) { *ok = true; return AEE_SUCCESS; }
  const size_t bytes = static_cast<size_t>(pq.view.n) * pq.view.dim * sizeof(float);
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  if (bytes > free_b / 2) return AEE_SUCCESS;
  if (pq.decoded.ensure(bytes) != cudaSuccess) {
    cudaGetLastError();
    return AEE_SUCCESS;
  }
  launch_pq_decode(pq.view, pq.decoded.as<float>(), s.stream);
  CK(cudaGetLastError());
  ++g_launches;
  CK(cudaStreamSynchronize(s.stream));
  pq.decoded_ready = true;
  *ok = true;
  return AEE_SUCCESS;
}

constexpr int kSharedVisitedSlots = 2048;             // per warp, 8 KB
constexpr size_t kSeedDistBudget = 512ull << 20;      // bytes of query x seed distances per launch

// Exact PQ search over decoded rows (pq_decoded.cu): per query chunk, the
// all-seeds distance pass, then the search kernel.
AEEResult pq_search_decoded(State& s, PqSearchArgs a, const RoverSearchParams* p, int nq, int expand,
                            cudaStream_t stream) {
  PqDevice& pq = s.pq;
  if (ensure_seeds(s, pq, p->entry_points, p->seed) != AEE_SUCCESS) return AEE_ENOMEMORY;
  // pools up to kVerifyMaxPool: TF32-ranked seeds verified exactly in the kernel;
  // wider pools: every seed's exact distance up front
  const bool verify = a.max_pool <= kVerifyMaxPool;
  if (verify && ensure_seed_drows(s, pq) != AEE_SUCCESS) return AEE_EFAILED;
  const SeedSet& ss = pq.seeds;
  PqDecodedArgs b{};
  b.decoded = pq.decoded.as<float>();
  b.seed_ids = ss.ids.as<int32_t>();
  b.n_seeds = ss.count;
  b.seed_dups = ss.dups;
  b.seed_bits = ss.bits.as<uint32_t>();
  b.seed_verify = verify ? 1 : 0;
  b.seed_norms = ss.drow_norms.as<float>();
  b.seed_norm_max = ss.drow_norm_max;
  b.seed_stride = verify ? (ss.count + 3) / 4 * 4 : ss.count;   // rank rows are read as float4
  pq_decoded_layout(&a, &b, p->refine_budget, kSharedVisitedSlots);
  const size_t slices = static_cast<size_t>(a.smem_per_warp) * kSearchWarps;
  if (slices > 227 * 1024) { set_error("shared memory %zu too large (pool %d)", slices, a.max_pool); return AEE_EBADPARM; }
  const PqDecodedFn kernel = pq_decoded_kernel_for(pq.view.dim);
  b.filter_bits = seed_filter_bits(reinterpret_cast<const void*>(kernel), kSearchWarps * 32, slices);
  const size_t smem = slices + static_cast<size_t>(b.filter_bits) / 8;
  if (allow_smem(reinterpret_cast<const void*>(kernel), smem) != AEE_SUCCESS) return AEE_EFAILED;
  const int max_blocks = resident_blocks(reinterpret_cast<const void*>(kernel), kSearchWarps * 32, smem, s.sms);
  const int chunk = static_cast<int>(std::max<size_t>(
      1, std::min<size_t>(nq, kSeedDistBudget / (static_cast<size_t>(b.seed_stride) * sizeof(float)))));
  CK(s.seed_dists.ensure(static_cast<size_t>(chunk) * b.seed_stride * sizeof(float)));
  b.seed_dists = s.seed_dists.as<float>();
  if (verify) {
    b.top_m = seed_top_m(ss.count, a.max_pool);
    CK(s.seed_top.ensure(static_cast<size_t>(chunk) * b.top_m * sizeof(uint64_t)));
    CK(s.seed_top_next.ensure(static_cast<size_t>(chunk) * sizeof(float)));
    b.seed_top = s.seed_top.as<uint64_t>();
    b.seed_top_next = s.seed_top_next.as<float>();
  }
  const int blocks_cap = std::max(1, std::min(max_blocks, (chunk + kSearchWarps - 1) / kSearchWarps));
  const size_t slots = static_cast<size_t>(blocks_cap) * kSearchWarps;
  uint32_t entries = next_pow2(std::max<uint64_t>(4096, 2 * (2ull * a.max_pool + 64ull) * expand));
  CK(s.counter.ensure(sizeof(unsigned int)));
  CK(cudaMemsetAsync(a.status, 0, nq * sizeof(int32_t), stream));
  for (int attempt = 0; attempt < 8; ++attempt) {
    uint32_t gen_base = 0;
    if (reserve_visited(s, slots, entries, static_cast<uint32_t>(nq), &gen_base) != AEE_SUCCESS) return AEE_ENOMEMORY;
    if (stream != s.stream) CK(cudaStreamSynchronize(s.stream));
    a.visited = s.visited.as<unsigned long long>();
    a.visited_mask = s.visited_mask;
    a.gen_base = gen_base;
    a.next_query = s.counter.as<unsigned int>();
    for (int q0 = 0; q0 < nq; q0 += chunk) {
      const int q1 = std::min(nq, q0 + chunk);
      if (verify) {
        if (ranked_seeds(s, stream, a.queries, q0, q1, pq.view.dim, ss.drows_map,
                         ss.drows_tc.p ? ss.drows_tc : ss.drows, ss.drow_norms, b.n_seeds, s.seed_dists.as<float>(),
                         b.seed_stride, b.top_m, s.seed_top.as<uint64_t>(), s.seed_top_next.as<float>()) !=
            AEE_SUCCESS)
          return AEE_EFAILED;
      } else {
        if (await_rows(s, stream, q1) != AEE_SUCCESS) return AEE_EFAILED;
        TimedLaunch tl(ROVER_KERNEL_PQ_SEEDS, stream);
        launch_pq_seed_dists(a.queries, q0, q1, pq.view.dim, b.decoded, b.seed_ids, b.n_seeds,
                             s.seed_dists.as<float>(), stream);
        ++g_launches;
      }
      CK(cudaGetLastError());
      if (await_rows(s, stream, q1) != AEE_SUCCESS) return AEE_EFAILED;
      b.q_begin = q0;
      b.q_end = q1;
      CK(cudaMemsetAsync(a.next_query, 0, sizeof(unsigned int), stream));
      const int blocks = std::max(1, std::min(blocks_cap, (q1 - q0 + kSearchWarps - 1) / kSearchWarps));
      {
        TimedLaunch tl(ROVER_KERNEL_PQ_DECODED, stream);
        kernel<<<blocks, kSearchWarps * 32, smem, stream>>>(a, b);
      }
      CK(cudaGetLastError());
      ++g_launches;
    }
    if (fetch_status(s, a.status, nq, stream) != AEE_SUCCESS) return AEE_EFAILED;
    collect_timings();
    if (check_tc_err(s) != AEE_SUCCESS) return AEE_EFAILED;
    bool retry = false;
    for (int i = 0; i < nq; ++i) retry |= s.h_status[i] == kStatusTableFull;
    if (!retry) break;
    entries = next_pow2(static_cast<uint64_t>(entries) * 4);
    CK(cudaMemsetAsync(a.status, 0, nq * sizeof(int32_t), stream));
  }
  for (int i = 0; i < nq; ++i)
    if (s.h_status[i] != kStatusOk) {
      set_error("query %d failed with status %d", i, s.h_status[i]);
      return AEE_EFAILED;
    }
  return AEE_SUCCESS;
}

AEEResult pq_search_batched(State& s, PqSearchArgs a, const RoverSearchParams* p, int nq, int expand,
                            cudaStream_t stream);

// Core PQ search on device buffers.  Retries queries whose visited table
// overflowed with a 4x larger table.
AEEResult pq_search_core(State& s, const RoverSearchParams* p, const float* d_queries, int nq,
                         const int32_t* d_pool, const int32_t* d_topk, const std::vector<int32_t>& h_pool,
                         const RoverSearchOutputs& d_out, cudaStream_t stream) {
  const PqDevice& pq = s.pq;
  if (!pq.loaded || !pq.has_graph) { set_error("no PQ index with a graph is loaded"); return AEE_EFAILED; }
  int max_pool = 0;
  for (int32_t v : h_pool) max_pool = std::max(max_pool, v);
  if (max_pool <= 0 || max_pool > 4096) { set_error("pool sizes must be in 1..4096"); return AEE_EBADPARM; }
  if (p->correction && pq.view.residual_bits == 0) { set_error("correction needs residuals"); return AEE_EBADPARM; }
  if (p->refine_budget > 0 && pq.view.residual_bits == 0) { set_error("refine needs residuals"); return AEE_EBADPARM; }
  if (p->third_residual && (!pq.view.e4.qparams || p->refine_budget <= 0)) {
    set_error("third_residual needs a loaded ERROR4 artifact and a refine budget");
    return AEE_EBADPARM;
  }
  const int expand = std::min(p->expand_count, pq.view.degree);
  if (expand > kMaxBatch) { set_error("expand_count above %d", kMaxBatch); return AEE_EBADPARM; }

  PqSearchArgs a{};
  a.ix = pq.view;
  a.queries = d_queries;
  a.nq = nq;
  a.pool_sizes = d_pool;
  a.top_ks = d_topk;
  a.top_k = p->top_k;
  a.entry_points = p->entry_points;
  a.graph_entry = pq.graph_entry;
  a.seed = p->seed;
  a.expand_count = p->expand_count;
  a.correction = p->correction;
  a.refine_budget = p->refine_budget;
  a.third_residual = p->third_residual;
  a.max_pool = max_pool;
  a.pool_ids = d_out.pool_ids;
  a.pool_dists = d_out.pool_dists;
  a.pool_stride = p->pool_stride;
  a.pool_counts = d_out.pool_counts;
  a.out_ids = d_out.ids;
  a.out_dists = d_out.dists;
  a.out_stride = d_out.out_stride;
  a.out_counts = d_out.counts;
  a.stats = reinterpret_cast<unsigned long long*>(d_out.stats);
  a.status = d_out.status;
  // residual layout: decoded rows when correction is on and they fit
  const bool decodable = p->correction != 0 && pq.view.dim % 4 == 0 &&
                         reinterpret_cast<uintptr_t>(d_queries) % 16 == 0;
  if (p->layout == ROVER_LAYOUT_DECODED && !decodable) {
    set_error("the decoded layout needs correction on, dim %% 4 == 0 and 16-byte aligned queries");
    return AEE_EBADPARM;
  }
  if (p->mode == ROVER_MODE_BATCHED || p->mode == ROVER_MODE_GATED || s.trace_dev) {
    if (!decodable || p->layout == ROVER_LAYOUT_PACKED) {
      set_error("batched and gated searches need correction on, decoded rows, dim %% 4 == 0 and aligned queries");
      return AEE_EBADPARM;
    }
    bool ok = false;
    if (ensure_decoded(s, s.pq, &ok) != AEE_SUCCESS) return AEE_EFAILED;
    if (!ok) { set_error("decoded rows do not fit in device memory"); return AEE_ENOMEMORY; }
    return pq_search_batched(s, a, p, nq, expand, stream);
  }
  if (p->mode != ROVER_MODE_EXACT) { set_error("unknown mode %d", p->mode); return AEE_EBADPARM; }
  if (decodable && p->layout != ROVER_LAYOUT_PACKED) {
    bool ok = false;
    if (ensure_decoded(s, s.pq, &ok) != AEE_SUCCESS) return AEE_EFAILED;
    if (ok) return pq_search_decoded(s, a, p, nq, expand, stream);
    if (p->layout == ROVER_LAYOUT_DECODED) { set_error("decoded rows do not fit in device memory"); return AEE_ENOMEMORY; }
  }
  pq_search_layout(&a, p->refine_budget);
  const size_t smem = static_cast<size_t>(a.smem_per_warp) * kSearchWarps;
  if (smem > 227 * 1024) { set_error("shared memory %zu too large (pool %d)", smem, max_pool); return AEE_EBADPARM; }
  const PqSearchFn kernel = pq_search_kernel_for(pq.view, p->correction != 0);
  if (allow_smem(reinterpret_cast<const void*>(kernel), smem) != AEE_SUCCESS) return AEE_EFAILED;
  const int max_blocks = resident_blocks(reinterpret_cast<const void*>(kernel), kSearchWarps * 32, smem, s.sms);
  const int blocks = std::max(1, std::min(max_blocks, (nq + kSearchWarps - 1) / kSearchWarps));
  const size_t slots = static_cast<size_t>(blocks) * kSearchWarps;
  const uint64_t est = static_cast<uint64_t>(std::min(p->entry_points, pq.view.n)) +
                       (2ull * max_pool + 64ull) * static_cast<uint64_t>(expand);
  uint32_t entries = next_pow2(std::max<uint64_t>(4096, 2 * est));
  CK(s.counter.ensure(sizeof(unsigned int)));
  CK(cudaMemsetAsync(d_out.status, 0, nq * sizeof(int32_t), stream));
  if (await_rows(s, stream, nq) != AEE_SUCCESS) return AEE_EFAILED;
  for (int attempt = 0; attempt < 8; ++attempt) {
    uint32_t gen_base = 0;
    if (reserve_visited(s, slots, entries, static_cast<uint32_t>(nq), &gen_base) != AEE_SUCCESS) return AEE_ENOMEMORY;
    if (stream != s.stream) {
      CK(cudaStreamSynchronize(s.stream));
    }
    a.visited = s.visited.as<unsigned long long>();
    a.visited_mask = s.visited_mask;
    a.gen_base = gen_base;
    a.next_query = s.counter.as<unsigned int>();
    CK(cudaMemsetAsync(a.next_query, 0, sizeof(unsigned int), stream));
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_PACKED, stream);
      kernel<<<blocks, kSearchWarps * 32, smem, stream>>>(a);
    }
    CK(cudaGetLastError());
    ++g_launches;
    if (fetch_status(s, d_out.status, nq, stream) != AEE_SUCCESS) return AEE_EFAILED;
    collect_timings();
    bool retry = false;
    for (int i = 0; i < nq; ++i) retry |= s.h_status[i] == kStatusTableFull;
    if (!retry) break;
    // Re-run everything with a larger table: the outputs of successful
    // queries are rewritten with identical values.
    entries = next_pow2(static_cast<uint64_t>(entries) * 4);
    CK(cudaMemsetAsync(d_out.status, 0, nq * sizeof(int32_t), stream));
  }
  for (int i = 0; i < nq; ++i)
    if (s.h_status[i] != kStatusOk) {
      set_error("query %d failed with status %d", i, s.h_status[i]);
      return AEE_EFAILED;
    }
  return AEE_SUCCESS;
}

// Batched / gated PQ search (pq_batched.cu): per query chunk, the
// all-seeds distance pass (not needed by the gate, which ranks seeds by ADC)
// and the batched kernel.  A trace request (s.trace_dev) records the gate's
// training rows.
AEEResult pq_search_batched(State& s, PqSearchArgs a, const RoverSearchParams* p, int nq, int expand,
                            cudaStream_t stream) {
  PqDevice& pq = s.pq;
  const bool tracing = s.trace_dev != nullptr;
  const bool gated = p->mode == ROVER_MODE_GATED && s.gate.enabled && !tracing;
  int W = tracing ? 1 : p->beam_width;
  if (W == 0) W = std::max(1, std::min(kMaxBeamWidth, kMaxBatchIds / std::max(1, expand)));
  if (expand > 2 * 32 || W < 1 || W > kMaxBeamWidth || W * expand > kMaxBatchIds) {
    set_error("batched search: need expand_count <= 64 and beam_width 1..%d with beam_width * expand_count <= %d",
              kMaxBeamWidth, kMaxBatchIds);
    return AEE_EBADPARM;
  }
  if (ensure_seeds(s, pq, p->entry_points, p->seed) != AEE_SUCCESS) return AEE_ENOMEMORY;
  const SeedSet& ss = pq.seeds;
  PqDecodedArgs b{};
  b.decoded = pq.decoded.as<float>();
  b.seed_ids = ss.ids.as<int32_t>();
  b.n_seeds = ss.count;
  b.seed_dups = ss.dups;
  b.seed_bits = ss.bits.as<uint32_t>();
  PqBatchArgs c{};
  c.beam_width = W;
  c.gate = s.gate;
  c.gate.enabled = gated ? 1 : 0;
  c.trace = s.trace_dev;
  c.trace_count = s.trace_count_dev;
  c.trace_cap = s.trace_cap;
  c.short_cap = 2 * a.max_pool;
  const bool rows = gated || tracing;   // seed ADC rows, shortlist and MLP scratch
  pq_batched_layout(&a, &b, &c, p->refine_budget, kSharedVisitedSlots, rows);
  const size_t slices = static_cast<size_t>(a.smem_per_warp) * kSearchWarps;
  if (slices > 227 * 1024) { set_error("shared memory %zu too large (pool %d)", slices, a.max_pool); return AEE_EBADPARM; }
  const PqBatchFn kernel = pq_batched_kernel_for(pq.view.dim, tracing ? kBatchTrace : gated ? kBatchGated : kBatchFull);
  b.filter_bits = seed_filter_bits(reinterpret_cast<const void*>(kernel), kSearchWarps * 32, slices);
  const size_t smem = slices + static_cast<size_t>(b.filter_bits) / 8;
  if (allow_smem(reinterpret_cast<const void*>(kernel), smem) != AEE_SUCCESS) return AEE_EFAILED;
  const int max_blocks = resident_blocks(reinterpret_cast<const void*>(kernel), kSearchWarps * 32, smem, s.sms);
  // exact seed pools: verified from TF32 ranks of the seeds' decoded rows
  // when every pool fits kVerifyMaxPool (as the exact decoded search does), else
  // the all-seeds exact distance pass
  const bool verify = !gated && !tracing && a.max_pool <= kVerifyMaxPool;
  const bool seed_pass = !gated && !verify;   // exact seed distances
  const bool rank_pass = rows;                // quantized seed distances (tensor cores)
  if (rank_pass && ensure_seed_recon(s, pq) != AEE_SUCCESS) return AEE_EFAILED;
  if (verify) {
    if (ensure_seed_drows(s, pq) != AEE_SUCCESS) return AEE_EFAILED;
    b.seed_verify = 1;
    b.seed_norms = ss.drow_norms.as<float>();
    b.seed_norm_max = ss.drow_norm_max;
    b.seed_stride = (ss.count + 3) / 4 * 4;   // rank rows are read as float4
    b.top_m = seed_top_m(ss.count, a.max_pool);
  }
  const size_t row_floats = verify ? static_cast<size_t>(b.seed_stride) : static_cast<size_t>(ss.count);
  // quantized rank rows padded to a multiple of 4 floats (vector stores)
  c.rank_stride = rank_pass ? (ss.count + 3) / 4 * 4 : 0;
  const size_t per_query = row_floats * sizeof(float) * (seed_pass || verify ? 1 : 0) +
                           static_cast<size_t>(c.rank_stride) * sizeof(float);
  const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(nq, kSeedDistBudget / per_query)));
  if (seed_pass || verify) CK(s.seed_dists.ensure(static_cast<size_t>(chunk) * row_floats * sizeof(float)));
  if (verify) {
    CK(s.seed_top.ensure(static_cast<size_t>(chunk) * b.top_m * sizeof(uint64_t)));
    CK(s.seed_top_next.ensure(static_cast<size_t>(chunk) * sizeof(float)));
    b.seed_top = s.seed_top.as<uint64_t>();
    b.seed_top_next = s.seed_top_next.as<float>();
  }
  if (rank_pass) {
    CK(s.seed_rank.ensure(static_cast<size_t>(chunk) * c.rank_stride * sizeof(float)));
    b.top_m = seed_top_m(ss.count, a.max_pool);
    CK(s.seed_top.ensure(static_cast<size_t>(chunk) * b.top_m * sizeof(uint64_t)));
    CK(s.seed_top_next.ensure(static_cast<size_t>(chunk) * sizeof(float)));
    b.seed_top = s.seed_top.as<uint64_t>();
    b.seed_top_next = s.seed_top_next.as<float>();
  }
  b.seed_dists = seed_pass || verify ? s.seed_dists.as<float>() : nullptr;
  c.seed_rank = rank_pass ? s.seed_rank.as<float>() : nullptr;
  const int blocks_cap = std::max(1, std::min(max_blocks, (chunk + kSearchWarps - 1) / kSearchWarps));
  const size_t slots = static_cast<size_t>(blocks_cap) * kSearchWarps;
  uint32_t entries = next_pow2(std::max<uint64_t>(4096, 2 * (2ull * a.max_pool + 64ull) * expand * W));
  CK(s.counter.ensure(sizeof(unsigned int)));
  CK(cudaMemsetAsync(a.status, 0, nq * sizeof(int32_t), stream));
  for (int attempt = 0; attempt < 8; ++attempt) {
    uint32_t gen_base = 0;
    if (reserve_visited(s, slots, entries, static_cast<uint32_t>(nq), &gen_base) != AEE_SUCCESS) return AEE_ENOMEMORY;
    if (stream != s.stream) CK(cudaStreamSynchronize(s.stream));
    if (tracing) CK(cudaMemsetAsync(s.trace_count_dev, 0, sizeof(unsigned long long), stream));
    a.visited = s.visited.as<unsigned long long>();
    a.visited_mask = s.visited_mask;
    a.gen_base = gen_base;
    a.next_query = s.counter.as<unsigned int>();
    for (int q0 = 0; q0 < nq; q0 += chunk) {
      const int q1 = std::min(nq, q0 + chunk);
      if (seed_pass) {
        if (await_rows(s, stream, q1) != AEE_SUCCESS) return AEE_EFAILED;
        {
          TimedLaunch tl(ROVER_KERNEL_PQ_SEEDS, stream);
          launch_pq_seed_dists(a.queries, q0, q1, pq.view.dim, b.decoded, b.seed_ids, b.n_seeds,
                               s.seed_dists.as<float>(), stream);
        }
        CK(cudaGetLastError());
        ++g_launches;
      }
      if (verify &&
          ranked_seeds(s, stream, a.queries, q0, q1, pq.view.dim, ss.drows_map,
                       ss.drows_tc.p ? ss.drows_tc : ss.drows, ss.drow_norms, b.n_seeds, s.seed_dists.as<float>(),
                       b.seed_stride, b.top_m, s.seed_top.as<uint64_t>(), s.seed_top_next.as<float>()) != AEE_SUCCESS)
        return AEE_EFAILED;
      if (rank_pass &&
          ranked_seeds(s, stream, a.queries, q0, q1, pq.view.dim, pq.seeds.recon_map,
                       pq.seeds.recon_tc.p ? pq.seeds.recon_tc : pq.seeds.recon, pq.seeds.recon_norms, b.n_seeds,
                       s.seed_rank.as<float>(), c.rank_stride, b.top_m, s.seed_top.as<uint64_t>(),
                       s.seed_top_next.as<float>()) != AEE_SUCCESS)
        return AEE_EFAILED;
      if (await_rows(s, stream, q1) != AEE_SUCCESS) return AEE_EFAILED;
      b.q_begin = q0;
      b.q_end = q1;
      CK(cudaMemsetAsync(a.next_query, 0, sizeof(unsigned int), stream));
      const int blocks = std::max(1, std::min(blocks_cap, (q1 - q0 + kSearchWarps - 1) / kSearchWarps));
      {
        TimedLaunch tl(ROVER_KERNEL_PQ_BATCHED, stream);
        kernel<<<blocks, kSearchWarps * 32, smem, stream>>>(a, b, c);
      }
      CK(cudaGetLastError());
      ++g_launches;
    }
    if (fetch_status(s, a.status, nq, stream) != AEE_SUCCESS) return AEE_EFAILED;
    collect_timings();
    if (check_tc_err(s) != AEE_SUCCESS) return AEE_EFAILED;
    bool retry = false;
    for (int i = 0; i < nq; ++i) retry |= s.h_status[i] == kStatusTableFull;
    if (!retry) break;
    entries = next_pow2(static_cast<uint64_t>(entries) * 4);
    CK(cudaMemsetAsync(a.status, 0, nq * sizeof(int32_t), stream));
  }
  for (int i = 0; i < nq; ++i)
    if (s.h_status[i] != kStatusOk) {
      set_error("query %d failed with status %d", i, s.h_status[i]);
      return AEE_EFAILED;
    }
  return AEE_SUCCESS;
}

template <class T>
AEEResult download(T* dst, const void* src, size_t count, cudaStream_t s) {
  if (dst && count) CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  return AEE_SUCCESS;
}

// The entry ids of an SQ search request, shared by its queries (they depend
// on the entry count, the graph entry and the seed only):
//  * DSP and DB-pair searches, dsp_search_select_entry_id
//    (retrieval_async_dsp_search.c:219): entry 0 is the graph entry when it is
//    valid, the others LCG draws from 42 scaled to [0, n); repeats stay in the
//    list (the search claims the first of each);
//  * SQMD, retrieval_sqmd_make_seed_ids (retrieval_sqmd_seed.c:15): the graph
//    entry, then (seed / 65536) % n LCG draws not yet in the list, at most
//    64 per wanted seed + 1024 draws, then the lowest ids not in it.
AEEResult sq_entries(State& s, SqDevice& sq, bool sqmd, int32_t entry_points, uint32_t seed) {
  const int32_t n = sq.view.n;
  const int32_t target = std::min(entry_points, n);
  if (sq.entries_valid && sq.entries_sqmd == sqmd && sq.entries_target == target && sq.entries_seed == seed)
    return AEE_SUCCESS;
  sq.entries_valid = false;
  std::vector<int32_t> ids;
  ids.reserve(static_cast<size_t>(std::max(target, 0)));
  const bool entry_ok = sq.graph_entry >= 0 && sq.graph_entry < n;
  if (!sqmd) {
    uint32_t lcg = 42u;
    for (int32_t i = 0; i < target; ++i) {
      if (i == 0 && entry_ok) {
        ids.push_back(sq.graph_entry);
        continue;
      }
      lcg = lcg * 1103515245u + 12345u;
      ids.push_back(static_cast<int32_t>((static_cast<uint64_t>(lcg) * static_cast<uint64_t>(n)) >> 32));
    }
  } else if (target > 0) {
    std::vector<uint8_t> taken(static_cast<size_t>(n), 0);
    auto take = [&](int32_t id) {
      if (taken[id]) return;
      taken[id] = 1;
      ids.push_back(id);
    };
    if (entry_ok) take(sq.graph_entry);
    const uint64_t limit = static_cast<uint64_t>(target) * 64u + 1024u;
    uint32_t lcg = seed;
    for (uint64_t attempts = 0; static_cast<int32_t>(ids.size()) < target && attempts < limit; ++attempts) {
      lcg = lcg * 1103515245u + 12345u;
      take(static_cast<int32_t>((lcg / 65536u) % static_cast<uint32_t>(n)));
    }
    for (int32_t id = 0; id < n && static_cast<int32_t>(ids.size()) < target; ++id) take(id);
  }
  if (ids.empty()) ids.push_back(-1);   // never read: entry_count is 0
  if (upload(sq.entry_ids, ids.data(), ids.size(), s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(cudaStreamSynchronize(s.stream));
  sq.entry_count = target > 0 ? static_cast<int32_t>(ids.size()) : 0;
  sq.entries_sqmd = sqmd;
  sq.entries_target = target;
  sq.entries_seed = seed;
  sq.entries_valid = true;
  return AEE_SUCCESS;
}

AEEResult sq_search_core(State& s, SqDevice& sq, int mode, const RoverSearchParams* p,
                         const float* d_queries, int nq, const int32_t* d_pool,
                         const std::vector<int32_t>& h_pool, int num_out, int32_t* d_ids, float* d_dists,
                         int32_t out_stride, int32_t* d_counts, unsigned long long* d_stats,
                         int32_t* d_status, cudaStream_t stream) {
  if (!sq.loaded) { set_error("no SQ index is loaded"); return AEE_EFAILED; }
  int max_pool = 0;
  for (int32_t v : h_pool) max_pool = std::max(max_pool, mode != kSqModeSqmd ? std::min(v, 2000) : v);
  if (max_pool <= 0 || max_pool > 4096) { set_error("pool sizes must be in 1..4096"); return AEE_EBADPARM; }
  const int expand = std::min(p->expand_count, sq.view.degree);
  const long long fbound = mode == kSqModeSqmd
                               ? static_cast<long long>(p->entry_points) + static_cast<long long>(max_pool) * p->expand_count
                               : static_cast<long long>(p->entry_points) + static_cast<long long>(max_pool) * expand;
  // the DB-pair search grows its frontier up to n entries: start at the
  // device search's bound and widen on a FRONTIER_FULL report
  int fcap = static_cast<int>(std::min<long long>(fbound, 1 << 20));
  if (mode == kSqModeDb) fcap = std::min(fcap, sq.view.n);
  SqSearchArgs a{};
  a.ix = sq.view;
  a.queries = d_queries;
  a.nq = nq;
  a.pool_sizes = d_pool;
  a.mode = mode;
  a.entry_points = p->entry_points;
  a.graph_entry = sq.graph_entry;
  a.seed = p->seed;
  a.expand_count = p->expand_count;
  a.correction = p->correction;
  a.split = p->split_distance;
  a.num_out = num_out;
  a.max_pool = max_pool;
  a.frontier_cap = fcap;
  a.out_ids = d_ids;
  a.out_dists = d_dists;
  a.out_stride = out_stride;
  a.out_counts = d_counts;
  a.stats = d_stats;
  a.status = d_status;
  if (sq_entries(s, sq, mode == kSqModeSqmd, p->entry_points, p->seed) != AEE_SUCCESS) return AEE_ENOMEMORY;
  a.entry_ids = sq.entry_ids.as<int32_t>();
  a.entry_count = sq.entry_count;
  // on-chip heap levels: with one block per SM enough for the batch, most of
  // the shared memory; otherwise a share that keeps four blocks per SM
  const bool few = nq <= s.sms * kSearchWarps;
  const size_t fixed = sq_search_smem_per_warp(sq.view.dim, 0, 0);
  const size_t budget = (few ? (200u << 10) : (48u << 10)) / kSearchWarps;
  const size_t room = budget > fixed ? (budget - fixed) / 8u : 0u;
  a.pool_split = static_cast<int32_t>(std::min<size_t>(static_cast<size_t>(max_pool), std::min<size_t>(room / 3u, few ? 1024u : 128u)));
  a.front_split = static_cast<int32_t>(std::min<size_t>(static_cast<size_t>(fcap), room - static_cast<size_t>(a.pool_split)));
  const size_t smem = sq_search_smem_per_warp(sq.view.dim, a.pool_split, a.front_split) * kSearchWarps;
  const SqSearchFn sq_kernel = sq_search_kernel_for(a.split != 0);
  if (allow_smem(reinterpret_cast<const void*>(sq_kernel), smem) != AEE_SUCCESS) return AEE_EFAILED;
  int blocks = std::max(1, std::min(resident_blocks(reinterpret_cast<const void*>(sq_kernel), kSearchWarps * 32, smem, s.sms),
                                    (nq + kSearchWarps - 1) / kSearchWarps));
  const int max_blocks = blocks;
  size_t slots = 0;
  // keep the heap scratch under 4 GiB
  auto size_heaps = [&]() -> AEEResult {
    const size_t heap_per_slot = static_cast<size_t>(max_pool + fcap) * 8u;
    blocks = max_blocks;
    while (blocks > 1 && static_cast<size_t>(blocks) * kSearchWarps * heap_per_slot > (4ull << 30)) blocks >>= 1;
    slots = static_cast<size_t>(blocks) * kSearchWarps;
    CK(s.heaps.ensure(slots * heap_per_slot));
    a.heaps = s.heaps.as<uint64_t>();
    a.frontier_cap = fcap;
    return AEE_SUCCESS;
  };
  if (size_heaps() != AEE_SUCCESS) return AEE_ENOMEMORY;
  const uint64_t est = static_cast<uint64_t>(p->entry_points) * 2 + (2ull * max_pool + 64ull) * static_cast<uint64_t>(std::max(expand, 1));
  uint32_t entries = next_pow2(std::max<uint64_t>(4096, 2 * est));
  CK(s.counter.ensure(sizeof(unsigned int)));
  CK(cudaMemsetAsync(d_status, 0, nq * sizeof(int32_t), stream));
  for (int attempt = 0; attempt < 8; ++attempt) {
    uint32_t gen_base = 0;
    if (reserve_visited(s, slots, entries, static_cast<uint32_t>(nq), &gen_base) != AEE_SUCCESS) return AEE_ENOMEMORY;
    a.visited = s.visited.as<unsigned long long>();
    a.visited_mask = s.visited_mask;
    a.gen_base = gen_base;
    a.next_query = s.counter.as<unsigned int>();
    CK(cudaMemsetAsync(a.next_query, 0, sizeof(unsigned int), stream));
    {
      TimedLaunch tl(ROVER_KERNEL_SQ, stream);
      sq_kernel<<<blocks, kSearchWarps * 32, smem, stream>>>(a);
    }
    CK(cudaGetLastError());
    ++g_launches;
    if (fetch_status(s, d_status, nq, stream) != AEE_SUCCESS) return AEE_EFAILED;
    collect_timings();
    bool retry = false, widen = false;
    for (int i = 0; i < nq; ++i) {
      retry |= s.h_status[i] == kStatusTableFull;
      widen |= mode == kSqModeDb && s.h_status[i] == kStatusFrontierFull && fcap < sq.view.n;
    }
    if (!retry && !widen) break;
    if (retry) entries = next_pow2(static_cast<uint64_t>(entries) * 4);
    if (widen) {
      fcap = static_cast<int>(std::min<long long>(4ll * fcap, sq.view.n));
      if (size_heaps() != AEE_SUCCESS) return AEE_ENOMEMORY;
    }
    CK(cudaMemsetAsync(d_status, 0, nq * sizeof(int32_t), stream));
  }
  for (int i = 0; i < nq; ++i)
    if (s.h_status[i] != kStatusOk) {
      set_error("query %d failed with status %d", i, s.h_status[i]);
      return AEE_EFAILED;
    }
  return AEE_SUCCESS;
}

AEEResult load_sq(State& s, SqDevice& d, const RoverSqIndexDesc* desc, int l1_bits) {
  if (!desc || desc->num_vectors <= 0 || desc->dim <= 0 || desc->dim > 1024 || desc->graph_degree <= 0 ||
      (l1_bits != 4 && l1_bits != 8) || !desc->l1_codes)
    return AEE_EBADPARM;
  d.release();
  const size_t n = desc->num_vectors;
  const int l1cb = l1_bits == 4 ? (desc->dim + 1) / 2 : desc->dim;
  if (desc->graph) {
    if (upload(d.graph, desc->graph, n * desc->graph_degree, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  }
  if (upload(d.l1, desc->l1_codes, n * l1cb, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  int rcb = 0;
  if (desc->residual_rows && desc->residual_qparams) {
    if (desc->residual_bits != 4 && desc->residual_bits != 8) return AEE_EBADPARM;
    rcb = desc->residual_bits == 4 ? (desc->dim + 1) / 2 : desc->dim;
    if (upload(d.residual, desc->residual_rows, n * rcb, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
    if (upload(d.qparams, desc->residual_qparams, n * 2, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  }
  CK(cudaStreamSynchronize(s.stream));
  SqIndexView& v = d.view;
  v.graph = d.graph.as<int32_t>();
  v.n = desc->num_vectors;
  v.degree = desc->graph_degree;
  v.dim = desc->dim;
  v.l1 = d.l1.as<uint8_t>();
  v.l1_bits = l1_bits;
  v.l1_code_bytes = l1cb;
  v.l1_scale = desc->l1_scale;
  v.l1_zero = desc->l1_zero;
  v.residual = rcb ? d.residual.as<uint8_t>() : nullptr;
  v.residual_bits = rcb ? desc->residual_bits : 0;
  v.rcb = rcb;
  v.qparams = rcb ? d.qparams.as<float>() : nullptr;
  d.graph_entry = desc->graph_entry;
  d.loaded = true;
  return AEE_SUCCESS;
}

}  // namespace

// ===========================================================================
// Extension entry points (include/rover_b200.h)

extern "C" const char* calculator_rover_last_error(void) { return g_last_error.c_str(); }

extern "C" uint64_t calculator_rover_launch_count(void) { return g_launches.load(); }

extern "C" void calculator_rover_kernel_timing(int32_t enable) {
  KernelTimer& t = timer();
  std::lock_guard<std::mutex> g(t.mu);
  t.on = enable != 0;
  for (int k = 0; k < ROVER_KERNEL_KINDS; ++k) {
    t.launches[k] = 0;
    t.ms[k] = 0.0;
  }
}

extern "C" int32_t calculator_rover_kernel_times(int64_t* launches, double* ms, int32_t kinds) {
  collect_timings();
  KernelTimer& t = timer();
  std::lock_guard<std::mutex> g(t.mu);
  const int32_t n = std::max(0, std::min<int32_t>(kinds, ROVER_KERNEL_KINDS));
  for (int32_t k = 0; k < n; ++k) {
    if (launches) launches[k] = t.launches[k];
    if (ms) ms[k] = t.ms[k];
  }
  return n;
}

extern "C" AEEResult calculator_rover_pq_load(remote_handle64 h, const RoverPqIndexDesc* d) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (session_busy(s, kSessionPurePq)) return AEE_EFAILED;
  if (!d || d->num_vectors <= 0 || d->dim <= 0 || d->dim > 1024 || d->m <= 0 ||
      (d->ks != 16 && d->ks != 256) || d->subdim <= 0 || d->m * d->subdim != d->dim ||
      d->code_bytes != (d->ks == 16 ? (d->m + 1) / 2 : d->m) || !d->codes || !d->codebook) {
    set_error("invalid PQ index description");
    return AEE_EBADPARM;
  }
  const size_t n = d->num_vectors;
  const size_t book = static_cast<size_t>(d->m) * d->ks * d->subdim;
  float absmax = 0.0f;
  for (size_t i = 0; i < book; ++i) {
    if (!std::isfinite(d->codebook[i])) { set_error("codebook is not finite"); return AEE_EBADPARM; }
    absmax = std::max(absmax, std::fabs(d->codebook[i]));
  }
  PqDevice& pq = s.pq;
  pq.release();
  AEEResult r = AEE_SUCCESS;
  if (d->graph) {
    if (d->graph_degree <= 0) return AEE_EBADPARM;
    r = upload(pq.graph, d->graph, n * d->graph_degree, s.stream);
    pq.has_graph = r == AEE_SUCCESS;
  }
  if (r == AEE_SUCCESS) r = upload(pq.codes, d->codes, n * d->code_bytes, s.stream);
  if (r == AEE_SUCCESS) r = upload(pq.codebook, d->codebook, book, s.stream);
  int rcb = 0, vpb = 0;
  if (r == AEE_SUCCESS && d->residual_bits) {
    if ((d->residual_bits != 4 && d->residual_bits != 8) || !d->residual_blocks || !d->residual_qparams) {
      set_error("invalid residual description");
      return AEE_EBADPARM;
    }
    rcb = d->residual_bits == 4 ? (d->dim + 1) / 2 : d->dim;
    vpb = 4096 / rcb;
    const int64_t blocks = (static_cast<int64_t>(n) + vpb - 1) / vpb;
    if (d->residual_blocks_bytes != blocks * 4096) {
      set_error("residual payload must be %lld bytes", static_cast<long long>(blocks * 4096));
      return AEE_EBADPARM;
    }
    r = upload(pq.residual, d->residual_blocks, static_cast<size_t>(d->residual_blocks_bytes), s.stream);
    if (r == AEE_SUCCESS) r = upload(pq.qparams, d->residual_qparams, n * 2, s.stream);
  }
  if (r != AEE_SUCCESS) { pq.release(); return AEE_ENOMEMORY; }
  CK(cudaStreamSynchronize(s.stream));
  PqIndexView& v = pq.view;
  v.graph = pq.graph.as<int32_t>();
  v.n = d->num_vectors;
  v.degree = d->graph ? d->graph_degree : 0;
  v.dim = d->dim;
  v.codes = pq.codes.as<uint8_t>();
  v.codebook = pq.codebook.as<float>();
  v.m = d->m;
  v.ks = d->ks;
  v.subdim = d->subdim;
  v.code_bytes = d->code_bytes;
  v.residual = rcb ? pq.residual.as<uint8_t>() : nullptr;
  v.residual_bits = rcb ? d->residual_bits : 0;
  v.rcb = rcb;
  v.vpb = vpb;
  v.qparams = rcb ? pq.qparams.as<float>() : nullptr;
  v.codebook_absmax = absmax;
  pq.graph_entry = d->graph_entry;
  pq.loaded = true;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_pq_unload(remote_handle64 h) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (session_busy(s, kSessionPurePq)) return AEE_EFAILED;
  s.pq.release();
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_pq_search_device(remote_handle64 h, const RoverSearchParams* p,
                                                       const float* queries, int32_t nq,
                                                       const int32_t* pool_sizes, const int32_t* top_ks,
                                                       const RoverSearchOutputs* out, void* stream) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!valid_params(p) || nq < 0 || !out || !queries || !pool_sizes || (out->ids && !out->counts)) return AEE_EBADPARM;
  if (nq == 0) return AEE_SUCCESS;
  cudaStream_t strm = stream ? static_cast<cudaStream_t>(stream) : s.stream;
  std::vector<int32_t> h_pool(nq);
  CK(cudaMemcpyAsync(h_pool.data(), pool_sizes, nq * sizeof(int32_t), cudaMemcpyDeviceToHost, strm));
  CK(cudaStreamSynchronize(strm));
  RoverSearchOutputs o = *out;
  if (!o.status) {
    CK(s.status.ensure(nq * sizeof(int32_t)));
    o.status = s.status.as<int32_t>();
  }
  return pq_search_core(s, p, queries, nq, pool_sizes, top_ks, h_pool, o, strm);
}

// Host-buffer PQ search (the lock is held by the caller).
AEEResult pq_search_host(State& s, const RoverSearchParams* p, const float* queries, int32_t nq,
                         const int32_t* pool_sizes, const int32_t* top_ks, const RoverSearchOutputs* out) {
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!valid_params(p) || nq < 0 || !out || !queries || !pool_sizes || (out->ids && !out->counts)) return AEE_EBADPARM;
  if (nq == 0) return AEE_SUCCESS;
  if (!s.pq.loaded) { set_error("no PQ index loaded"); return AEE_EFAILED; }
  cudaStream_t strm = s.stream;
  const int dim = s.pq.view.dim;
  std::vector<int32_t> h_pool(pool_sizes, pool_sizes + nq);
  int max_pool = 0;
  for (int v : h_pool) max_pool = std::max(max_pool, v);
  const int k_stride = out->ids ? out->out_stride : 0;
  const int p_stride = out->pool_ids ? p->pool_stride : 0;
  // Large batches upload their queries in four pieces on the copy stream;
  // the seed ranking of each piece starts when it has arrived (await_rows),
  // so the upload overlaps the seed pass.
  struct ArrivalScope {
    State& s;
    ~ArrivalScope() {
      if (s.arrival_pieces) cudaStreamSynchronize(s.copy_stream);   // no copy from the caller's memory outlives the call
      s.arrival_pieces = 0;
    }
  } arrival{s};
  const int pieces = nq >= 2048 && s.copy_stream ? 4 : 1;
  if (pieces > 1) {
    const size_t bytes = static_cast<size_t>(nq) * dim * sizeof(float);
    CK(s.in_queries.ensure(bytes));
    const int rows = (((nq + pieces - 1) / pieces) + 127) / 128 * 128;   // whole 128-query tiles of the ranking
    int k = 0;
    for (int q0 = 0; q0 < nq; q0 += rows, ++k) {
      const size_t n = static_cast<size_t>(std::min(nq, q0 + rows) - q0) * dim;
      CK(cudaMemcpyAsync(s.in_queries.as<float>() + static_cast<size_t>(q0) * dim,
                         queries + static_cast<size_t>(q0) * dim, n * sizeof(float), cudaMemcpyHostToDevice,
                         s.copy_stream));
      CK(cudaEventRecord(s.arrival_ev[k], s.copy_stream));
    }
    s.arrival_rows = rows;
    s.arrival_pieces = k;
  } else if (upload(s.in_queries, queries, static_cast<size_t>(nq) * dim, strm) != AEE_SUCCESS) {
    return AEE_ENOMEMORY;
  }
  if (upload(s.in_pool, pool_sizes, nq, strm) != AEE_SUCCESS) return AEE_ENOMEMORY;
  if (top_ks && upload(s.in_topk, top_ks, nq, strm) != AEE_SUCCESS) return AEE_ENOMEMORY;
  RoverSearchOutputs d{};
  if (k_stride) {
    CK(s.out_ids.ensure(static_cast<size_t>(nq) * k_stride * 4));
    CK(s.out_dists.ensure(static_cast<size_t>(nq) * k_stride * 4));
    CK(s.out_counts.ensure(static_cast<size_t>(nq) * 4));
    d.ids = s.out_ids.as<int32_t>();
    d.dists = s.out_dists.as<float>();
    d.counts = s.out_counts.as<int32_t>();
    d.out_stride = k_stride;
  }
  if (p_stride) {
    CK(s.pool_ids.ensure(static_cast<size_t>(nq) * p_stride * 4));
    CK(s.pool_dists.ensure(static_cast<size_t>(nq) * p_stride * 4));
    CK(s.pool_counts.ensure(static_cast<size_t>(nq) * 4));
    d.pool_ids = s.pool_ids.as<int32_t>();
    d.pool_dists = s.pool_dists.as<float>();
    d.pool_counts = s.pool_counts.as<int32_t>();
  }
  if (out->stats) {
    CK(s.stats.ensure(static_cast<size_t>(nq) * 32));
    d.stats = s.stats.as<uint64_t>();
  }
  CK(s.status.ensure(static_cast<size_t>(nq) * 4));
  d.status = s.status.as<int32_t>();
  RoverSearchParams pp = *p;
  pp.pool_stride = p_stride;
  ResultStage rs(s);
  const size_t nk = static_cast<size_t>(nq) * k_stride, np = static_cast<size_t>(nq) * p_stride;
  if (k_stride) {
    rs.add(out->ids, d.ids, nk * sizeof(int32_t));
    rs.add(out->dists, d.dists, nk * sizeof(float));
    rs.add(out->counts, d.counts, static_cast<size_t>(nq) * sizeof(int32_t));
  }
  if (p_stride) {
    rs.add(out->pool_ids, d.pool_ids, np * sizeof(int32_t));
    rs.add(out->pool_dists, d.pool_dists, np * sizeof(float));
    rs.add(out->pool_counts, d.pool_counts, static_cast<size_t>(nq) * sizeof(int32_t));
  }
  if (out->stats) rs.add(out->stats, d.stats, static_cast<size_t>(nq) * 4 * sizeof(uint64_t));
  if (rs.arm() != AEE_SUCCESS) return AEE_ENOMEMORY;
  AEEResult r = pq_search_core(s, &pp, s.in_queries.as<float>(), nq, s.in_pool.as<int32_t>(),
                               top_ks ? s.in_topk.as<int32_t>() : nullptr, h_pool, d, strm);
  if (out->status) {
    std::copy(s.h_status.begin(), s.h_status.begin() + nq, out->status);
  }
  if (r != AEE_SUCCESS) return r;
  return rs.finish(strm);
}

extern "C" AEEResult calculator_rover_pq_search(remote_handle64 h, const RoverSearchParams* p,
                                                const float* queries, int32_t nq, const int32_t* pool_sizes,
                                                const int32_t* top_ks, const RoverSearchOutputs* out) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  return pq_search_host(s, p, queries, nq, pool_sizes, top_ks, out);
}

// ---------------------------------------------------------------------------
// Search plans (include/rover_b200.h): a fixed kernel sequence over a fixed
// set of beam widths and result counts, enqueued without allocation or host
// waits so that one launch can be captured into a CUDA graph and replayed.

struct RoverPqPlan {};   // the opaque handle type of the C-ABI
static_assert(ROVER_PLAN_MAX_CLASSES == rover::kMaxPlanClasses, "plan classes");

namespace {

constexpr uint32_t kPlanMagic = 0x4e414c50u;
constexpr int32_t kPlanMaxQueries = 4000000;          // seed passes tile queries by 64 in grid.y
constexpr size_t kPlanSeedBytes = 8ull << 30;          // query x seed distances held by one plan

struct PlanConfig {
  int layout = ROVER_LAYOUT_DECODED;
  int warps = kSearchWarps;
  int vis_cap = kSharedVisitedSlots;
  int split = 0;            // 0: one class, 1: two classes, 2: one class per power of two of L
};

struct PlanClass {
  int offset = 0, count = 0, max_pool = 0, blocks = 0;
  uint32_t entries = 0;     // visited-table entries per warp slot
  size_t smem = 0;          // per CTA: seed filter + warp slices
  int filter_bits = 0;      // seed filter (decoded and batched kernels)
};

struct PqPlanImpl : RoverPqPlan {
  uint32_t magic = kPlanMagic;
  uint64_t epoch = 0;                   // PqDevice::epoch of the index the plan was made on
  RoverSearchParams p{};
  int nq = 0, expand = 0, max_pool = 0, max_k = 0, W = 1;
  bool gated = false, has_topk = false;
  bool decodable = false;               // decoded rows available for this request
  bool allow_packed = false, allow_decoded = false;
  PlanConfig cfg;
  std::vector<PlanClass> classes;
  std::vector<int32_t> h_pool, h_order;
  uint32_t table_scale = 1;             // visited tables grown after an overflow while tuning
  size_t visited_words = 0;
  int candidates = 0;
  float tuned_ms = 0.0f, default_ms = 0.0f;
  int32_t n_seeds = 0, seed_dups = 0;
  GateParams gate{};
  DevBuf pool, topk, order, ctl, visited, seed_ids, seed_bits, recon, recon_norms, seed_dists, seed_rank, gate_buf;
  DevBuf drows, drow_norms;             // exact plans: the seeds' decoded rows for the verified seed pool
  // TF32-rounded copies of drows / recon named by TMA descriptors: the
  // plan ranks its seeds on the tensor cores (valid == 0: mma.sync)
  DevBuf drows_tc, recon_tc;
  TcSeedMap drows_map{}, recon_map{};
  DevBuf seed_top, seed_top_next;       // per query: top-M seed ranks (verified and gated plans)
  int32_t top_m = 0;
  bool verify_seeds = false;            // exact / batched decoded plan, every pool <= kVerifyMaxPool
  int32_t seed_stride = 0;              // floats per query row of seed_dists
  float drow_norm_max = 0.0f;
  size_t device_bytes() const {
    return pool.bytes + topk.bytes + order.bytes + ctl.bytes + visited.bytes + seed_ids.bytes + seed_bits.bytes +
           recon.bytes + recon_norms.bytes + seed_dists.bytes + seed_rank.bytes + gate_buf.bytes + drows.bytes +
           drow_norms.bytes + seed_top.bytes + seed_top_next.bytes;
  }
  void release() {
    for (DevBuf* b : {&pool, &topk, &order, &ctl, &visited, &seed_ids, &seed_bits, &recon, &recon_norms, &seed_dists,
                      &seed_rank, &gate_buf, &drows, &drow_norms, &seed_top, &seed_top_next})
      b->release();
  }
};

PqPlanImpl* plan_cast(const RoverPqPlan* p) {
  auto* q = static_cast<PqPlanImpl*>(const_cast<RoverPqPlan*>(p));
  return q && q->magic == kPlanMagic ? q : nullptr;
}

uint32_t ceil_pow2_log(int v) {
  uint32_t l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

// Beam-width classes over the plan's order (widest first).  split 1 picks
// the power-of-two boundary that minimises the shared memory the queries'
// slices take (count x widest width of the class); split 2 gives each power
// of two its own class (the narrowest merged down to kMaxPlanClasses).
std::vector<PlanClass> plan_classes(const PqPlanImpl& P, int split) {
  const int nq = P.nq;
  std::vector<PlanClass> out;
  auto add = [&](int off, int cnt) {
    PlanClass c;
    c.offset = off;
    c.count = cnt;
    c.max_pool = P.h_pool[P.h_order[off]];
    out.push_back(c);
  };
  if (split == 0) {
    add(0, nq);
    return out;
  }
  std::vector<uint32_t> key(nq);
  const uint32_t top = ceil_pow2_log(P.h_pool[P.h_order[0]]);
  for (int j = 0; j < nq; ++j) {
    const uint32_t k = ceil_pow2_log(P.h_pool[P.h_order[j]]);
    key[j] = std::max(k, top >= kMaxPlanClasses - 1 ? top - (kMaxPlanClasses - 1) : 0u);
  }
  if (split == 2) {
    int off = 0;
    for (int j = 1; j <= nq; ++j)
      if (j == nq || key[j] != key[off]) {
        add(off, j - off);
        off = j;
      }
    return out;
  }
  // split 1: one boundary between consecutive keys
  int best_cut = nq;
  double best_cost = static_cast<double>(nq) * P.h_pool[P.h_order[0]];
  for (int j = 1; j < nq; ++j) {
    if (key[j] == key[j - 1]) continue;
    const double cost = static_cast<double>(j) * P.h_pool[P.h_order[0]] +
                        static_cast<double>(nq - j) * P.h_pool[P.h_order[j]];
    if (cost < best_cost) { best_cost = cost; best_cut = j; }
  }
  add(0, best_cut);
  if (best_cut < nq) add(best_cut, nq - best_cut);
  return out;
}

// Arguments shared by every search launch of a plan.
PqSearchArgs plan_args(const State& s, const PqPlanImpl& P, const float* queries, const RoverSearchOutputs& o) {
  const PqDevice& pq = s.pq;
  PqSearchArgs a{};
  a.ix = pq.view;
  a.queries = queries;
  a.nq = P.nq;
  a.pool_sizes = P.pool.as<int32_t>();
  a.top_ks = P.has_topk ? P.topk.as<int32_t>() : nullptr;
  a.top_k = P.p.top_k;
  a.entry_points = P.p.entry_points;
  a.graph_entry = pq.graph_entry;
  a.seed = P.p.seed;
  a.expand_count = P.p.expand_count;
  a.correction = P.p.correction;
  a.refine_budget = P.p.refine_budget;
  a.third_residual = P.p.third_residual;
  a.max_pool = P.max_pool;
  a.pool_ids = o.pool_ids;
  a.pool_dists = o.pool_dists;
  a.pool_stride = o.pool_ids ? P.p.pool_stride : 0;
  a.pool_counts = o.pool_counts;
  a.out_ids = o.ids;
  a.out_dists = o.dists;
  a.out_stride = o.out_stride;
  a.out_counts = o.counts;
  a.stats = reinterpret_cast<unsigned long long*>(o.stats);
  a.status = o.status;
  a.visited = P.visited.as<unsigned long long>();
  a.gen_dev = &P.ctl.as<PlanControl>()->gen;
  a.order = P.order.as<int32_t>();
  return a;
}

PqDecodedArgs plan_decoded_args(const State& s, const PqPlanImpl& P) {
  PqDecodedArgs b{};
  b.decoded = s.pq.decoded.as<float>();
  b.seed_ids = P.seed_ids.as<int32_t>();
  b.n_seeds = P.n_seeds;
  b.seed_dups = P.seed_dups;
  b.seed_bits = P.seed_bits.as<uint32_t>();
  b.seed_dists = P.seed_dists.as<float>();
  b.seed_verify = P.verify_seeds ? 1 : 0;
  b.seed_norms = P.drow_norms.as<float>();
  b.seed_norm_max = P.drow_norm_max;
  b.seed_stride = P.seed_stride;
  if (P.top_m) {
    b.seed_top = P.seed_top.as<uint64_t>();
    b.seed_top_next = P.seed_top_next.as<float>();
    b.top_m = P.top_m;
  }
  if (P.drows_map.valid || P.recon_map.valid) b.seed_err = s.tc_err.as<int>();
  return b;
}

PqBatchArgs plan_batch_args(const PqPlanImpl& P) {
  PqBatchArgs c{};
  c.beam_width = P.W;
  c.gate = P.gate;
  c.gate.enabled = P.gated ? 1 : 0;
  c.seed_rank = P.gated ? P.seed_rank.as<float>() : nullptr;
  return c;
}

const void* plan_kernel(const State& s, const PqPlanImpl& P, int layout) {
  const PqDevice& pq = s.pq;
  if (layout == ROVER_LAYOUT_PACKED)
    return reinterpret_cast<const void*>(pq_search_kernel_for(pq.view, P.p.correction != 0));
  if (P.p.mode == ROVER_MODE_EXACT) return reinterpret_cast<const void*>(pq_decoded_kernel_for(pq.view.dim));
  return reinterpret_cast<const void*>(pq_batched_kernel_for(pq.view.dim, P.gated ? kBatchGated : kBatchFull));
}

// Shared-memory slice layout of one class (a.max_pool set to its widest beam).
void plan_layout(const PqPlanImpl& P, int layout, int vis_cap, PqSearchArgs* a, PqDecodedArgs* b, PqBatchArgs* c) {
  if (layout == ROVER_LAYOUT_PACKED) {
    pq_search_layout(a, P.p.refine_budget);
  } else if (P.p.mode == ROVER_MODE_EXACT) {
    pq_decoded_layout(a, b, P.p.refine_budget, vis_cap);
  } else {
    c->short_cap = 2 * a->max_pool;
    pq_batched_layout(a, b, c, P.p.refine_budget, vis_cap, P.gated);
  }
}

// Fixes the classes, launch shapes and visited tables of a configuration.
// Returns AEE_EBADPARM (with nothing changed) when a slice does not fit.
AEEResult plan_configure(State& s, PqPlanImpl& P, const PlanConfig& cfg) {
  const PqDevice& pq = s.pq;
  const int warps = cfg.layout == ROVER_LAYOUT_PACKED ? kSearchWarps : cfg.warps;
  std::vector<PlanClass> cls = plan_classes(P, cfg.split);
  const void* kernel = plan_kernel(s, P, cfg.layout);
  size_t words = 0, smem_max = 0;
  for (PlanClass& c : cls) {
    PqSearchArgs a{};
    a.ix = pq.view;
    a.max_pool = c.max_pool;
    PqDecodedArgs b{};
    PqBatchArgs bc{};
    bc.beam_width = P.W;
    plan_layout(P, cfg.layout, cfg.vis_cap, &a, &b, &bc);
    const size_t slices = static_cast<size_t>(a.smem_per_warp) * warps;
    if (slices > 227 * 1024) return AEE_EBADPARM;
    c.filter_bits = cfg.layout == ROVER_LAYOUT_PACKED ? 0 : seed_filter_bits(kernel, warps * 32, slices);
    c.smem = slices + static_cast<size_t>(c.filter_bits) / 8;
    smem_max = std::max(smem_max, c.smem);
  }
  if (allow_smem(kernel, smem_max) != AEE_SUCCESS) return AEE_EFAILED;
  for (PlanClass& c : cls) {
    const int max_blocks = resident_blocks(kernel, warps * 32, c.smem, s.sms);
    c.blocks = std::max(1, std::min(max_blocks, (c.count + warps - 1) / warps));
    uint64_t est = (2ull * c.max_pool + 64ull) * static_cast<uint64_t>(P.expand);
    if (cfg.layout == ROVER_LAYOUT_PACKED) est += static_cast<uint64_t>(std::min(P.p.entry_points, pq.view.n));
    else est *= static_cast<uint64_t>(P.W);
    c.entries = next_pow2(std::max<uint64_t>(4096, 2 * est) * P.table_scale);
    words = std::max(words, static_cast<size_t>(c.blocks) * warps * c.entries);
  }
  if (words * 8 > P.visited.bytes) {
    // fresh memory may hold anything a live tag could match: zero it
    P.visited.release();
    CK(P.visited.ensure(words * 8));
    CK(cudaMemsetAsync(P.visited.p, 0, words * 8, s.stream));
    CK(cudaStreamSynchronize(s.stream));
  }
  P.cfg = cfg;
  P.cfg.warps = warps;
  P.classes = cls;
  P.visited_words = words;
  return AEE_SUCCESS;
}

bool stream_capturing(cudaStream_t stream) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs != cudaStreamCaptureStatusNone;
}

// The kernels of one plan launch.  No allocation, no host synchronisation.
AEEResult plan_enqueue(State& s, PqPlanImpl& P, const float* queries, const RoverSearchOutputs& o,
                       cudaStream_t stream) {
  const PqDevice& pq = s.pq;
  const bool timed = !stream_capturing(stream);
  PlanControl* ctl = P.ctl.as<PlanControl>();
  const int nclass = static_cast<int>(P.classes.size());
  {
    TimedLaunch tl(ROVER_KERNEL_PLAN, stream, timed);
    launch_plan_prepare(ctl, P.visited.as<unsigned long long>(), P.visited_words, o.status, P.nq, nclass, s.sms,
                        stream);
  }
  CK(cudaGetLastError());
  ++g_launches;
  const bool decoded = P.cfg.layout != ROVER_LAYOUT_PACKED;
  // seed ranks on the tensor cores when the rows have a descriptor
  auto rank = [&](const TcSeedMap& map, const DevBuf& rows, const DevBuf& norms, float* out, int stride) {
    if (map.valid && launch_pq_seed_rank_tc(map, queries, 0, P.nq, pq.view.dim, norms.as<float>(), P.n_seeds, out,
                                            stride, s.tc_err.as<int>(), s.sms, stream))
      return;
    launch_pq_seed_rank(queries, 0, P.nq, pq.view.dim, rows.as<float>(), norms.as<float>(), P.n_seeds, out, stream,
                        stride);
  };
  if (decoded && P.verify_seeds) {
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEED_RANK, stream, timed);
      rank(P.drows_map, P.drows, P.drow_norms, P.seed_dists.as<float>(), P.seed_stride);
    }
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEED_TOPM, stream, timed);
      launch_pq_seed_topm(P.seed_dists.as<float>(), P.seed_stride, P.n_seeds, P.nq, P.top_m,
                          P.seed_top.as<uint64_t>(), P.seed_top_next.as<float>(), stream);
    }
    CK(cudaGetLastError());
    g_launches += 2;
  } else if (decoded && !P.gated) {
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEEDS, stream, timed);
      launch_pq_seed_dists(queries, 0, P.nq, pq.view.dim, pq.decoded.as<float>(), P.seed_ids.as<int32_t>(),
                           P.n_seeds, P.seed_dists.as<float>(), stream);
    }
    CK(cudaGetLastError());
    ++g_launches;
  }
  if (decoded && P.gated) {
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEED_RANK, stream, timed);
      rank(P.recon_map, P.recon, P.recon_norms, P.seed_rank.as<float>(), P.n_seeds);
    }
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_SEED_TOPM, stream, timed);
      launch_pq_seed_topm(P.seed_rank.as<float>(), P.n_seeds, P.n_seeds, P.nq, P.top_m, P.seed_top.as<uint64_t>(),
                          P.seed_top_next.as<float>(), stream);
    }
    CK(cudaGetLastError());
    g_launches += 2;
  }
  const void* kernel = plan_kernel(s, P, P.cfg.layout);
  const int threads = P.cfg.warps * 32;
  for (int ci = 0; ci < nclass; ++ci) {
    const PlanClass& c = P.classes[ci];
    PqSearchArgs a = plan_args(s, P, queries, o);
    a.max_pool = c.max_pool;
    a.visited_mask = c.entries - 1u;
    a.next_query = &ctl->counters[ci];
    PqDecodedArgs b = plan_decoded_args(s, P);
    PqBatchArgs bc = plan_batch_args(P);
    plan_layout(P, P.cfg.layout, P.cfg.vis_cap, &a, &b, &bc);
    b.filter_bits = c.filter_bits;
    if (!decoded) {
      a.order = P.order.as<int32_t>() + c.offset;
      a.nq = c.count;
      TimedLaunch tl(ROVER_KERNEL_PQ_PACKED, stream, timed);
      reinterpret_cast<PqSearchFn>(const_cast<void*>(kernel))<<<c.blocks, threads, c.smem, stream>>>(a);
    } else if (P.p.mode == ROVER_MODE_EXACT) {
      b.q_begin = c.offset;
      b.q_end = c.offset + c.count;
      TimedLaunch tl(ROVER_KERNEL_PQ_DECODED, stream, timed);
      reinterpret_cast<PqDecodedFn>(const_cast<void*>(kernel))<<<c.blocks, threads, c.smem, stream>>>(a, b);
    } else {
      b.q_begin = c.offset;
      b.q_end = c.offset + c.count;
      TimedLaunch tl(ROVER_KERNEL_PQ_BATCHED, stream, timed);
      reinterpret_cast<PqBatchFn>(const_cast<void*>(kernel))<<<c.blocks, threads, c.smem, stream>>>(a, b, bc);
    }
    CK(cudaGetLastError());
    ++g_launches;
  }
  {
    TimedLaunch tl(ROVER_KERNEL_PLAN, stream, timed);
    launch_plan_advance(ctl, P.nq, stream);
  }
  CK(cudaGetLastError());
  ++g_launches;
  return AEE_SUCCESS;
}

// Times one configuration on the tuning queries (best of `reps` launches
// after one warm-up).  *overflow reports a visited-table overflow.
AEEResult plan_time(State& s, PqPlanImpl& P, const float* queries, const RoverSearchOutputs& o, int reps,
                    float* best_ms, bool* overflow) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    set_error("cudaEventCreate failed");
    return AEE_EFAILED;
  }
  AEEResult r = AEE_SUCCESS;
  float best = 0.0f;
  for (int rep = 0; rep <= reps && r == AEE_SUCCESS; ++rep) {
    cudaEventRecord(e0, s.stream);
    r = plan_enqueue(s, P, queries, o, s.stream);
    cudaEventRecord(e1, s.stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      set_error("plan launch failed: %s", cudaGetErrorString(cudaGetLastError()));
      r = AEE_EFAILED;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best == 0.0f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  collect_timings();
  if (r != AEE_SUCCESS) return r;
  s.h_status.resize(P.nq);
  CK(cudaMemcpy(s.h_status.data(), o.status, P.nq * sizeof(int32_t), cudaMemcpyDeviceToHost));
  *overflow = false;
  for (int i = 0; i < P.nq; ++i) *overflow |= s.h_status[i] == kStatusTableFull;
  *best_ms = best;
  return AEE_SUCCESS;
}

// Copies the entry seeds (and for gated plans their reconstructions and the
// loaded gate) into plan-owned buffers and sizes the seed-pass outputs.
AEEResult plan_inputs(State& s, PqPlanImpl& P) {
  PqDevice& pq = s.pq;
  if (ensure_seeds(s, pq, P.p.entry_points, P.p.seed) != AEE_SUCCESS) return AEE_ENOMEMORY;
  const SeedSet& ss = pq.seeds;
  P.n_seeds = ss.count;
  P.seed_dups = ss.dups;
  const size_t bits_bytes = (static_cast<size_t>(pq.view.n) + 31) / 32 * 4;
  CK(P.seed_ids.ensure(static_cast<size_t>(ss.count) * 4));
  CK(P.seed_bits.ensure(bits_bytes));
  CK(cudaMemcpyAsync(P.seed_ids.p, ss.ids.p, static_cast<size_t>(ss.count) * 4, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaMemcpyAsync(P.seed_bits.p, ss.bits.p, bits_bytes, cudaMemcpyDeviceToDevice, s.stream));
  if (!P.allow_decoded) return AEE_SUCCESS;
  P.verify_seeds = (P.p.mode == ROVER_MODE_EXACT || P.p.mode == ROVER_MODE_BATCHED) &&
                  P.max_pool <= kVerifyMaxPool && !P.gated;
  P.seed_stride = P.verify_seeds ? (ss.count + 3) / 4 * 4 : ss.count;
  const size_t seed_bytes = static_cast<size_t>(P.nq) * P.seed_stride * sizeof(float);
  if (seed_bytes > kPlanSeedBytes) {
    set_error("a plan of %d queries x %d seeds needs %zu bytes of seed distances (limit %zu): use smaller plans",
              P.nq, ss.count, seed_bytes, kPlanSeedBytes);
    return AEE_EBADPARM;
  }
  if (P.gated || P.verify_seeds) {
    P.top_m = seed_top_m(ss.count, P.max_pool);
    CK(P.seed_top.ensure(static_cast<size_t>(P.nq) * P.top_m * sizeof(uint64_t)));
    CK(P.seed_top_next.ensure(static_cast<size_t>(P.nq) * sizeof(float)));
  }
  if (P.gated) {
    if (ensure_seed_recon(s, pq) != AEE_SUCCESS) return AEE_EFAILED;
    const size_t rb = static_cast<size_t>(ss.count) * pq.view.dim * sizeof(float);
    CK(P.recon.ensure(rb));
    CK(P.recon_norms.ensure(static_cast<size_t>(ss.count) * sizeof(float)));
    CK(cudaMemcpyAsync(P.recon.p, ss.recon.p, rb, cudaMemcpyDeviceToDevice, s.stream));
    CK(cudaMemcpyAsync(P.recon_norms.p, ss.recon_norms.p, static_cast<size_t>(ss.count) * sizeof(float),
                       cudaMemcpyDeviceToDevice, s.stream));
    // (gated plans keep the mma.sync ranking: inside a plan the tcgen05 ranking
    // of the reconstructions measured 0.52 ms against 0.29 ms on mma.sync per
    // 10,000 queries x 8,192 seeds, for a cause not found yet)
    CK(P.seed_rank.ensure(seed_bytes));
    // the gate's weights move with the plan: rebase its pointers
    CK(P.gate_buf.ensure(s.gate_buf.bytes));
    CK(cudaMemcpyAsync(P.gate_buf.p, s.gate_buf.p, s.gate_buf.bytes, cudaMemcpyDeviceToDevice, s.stream));
    auto rebase = [&](const void* q) {
      return static_cast<const uint8_t*>(P.gate_buf.p) +
             (static_cast<const uint8_t*>(q) - static_cast<const uint8_t*>(s.gate_buf.p));
    };
    P.gate = s.gate;
    P.gate.w1t = reinterpret_cast<const uint16_t*>(rebase(s.gate.w1t));
    P.gate.w2t = reinterpret_cast<const uint16_t*>(rebase(s.gate.w2t));
    P.gate.w3t = reinterpret_cast<const uint16_t*>(rebase(s.gate.w3t));
    P.gate.b1 = reinterpret_cast<const float*>(rebase(s.gate.b1));
    P.gate.b2 = reinterpret_cast<const float*>(rebase(s.gate.b2));
    P.gate.b3 = reinterpret_cast<const float*>(rebase(s.gate.b3));
    P.gate.rows_evaluated = reinterpret_cast<unsigned long long*>(
        const_cast<void*>(static_cast<const void*>(rebase(s.gate.rows_evaluated))));
  } else {
    CK(P.seed_dists.ensure(seed_bytes));
    if (P.verify_seeds) {
      if (ensure_seed_drows(s, pq) != AEE_SUCCESS) return AEE_EFAILED;
      const size_t rb = static_cast<size_t>(ss.count) * pq.view.dim * sizeof(float);
      CK(P.drows.ensure(rb));
      CK(P.drow_norms.ensure(static_cast<size_t>(ss.count) * sizeof(float)));
      CK(cudaMemcpyAsync(P.drows.p, ss.drows.p, rb, cudaMemcpyDeviceToDevice, s.stream));
      CK(cudaMemcpyAsync(P.drow_norms.p, ss.drow_norms.p, static_cast<size_t>(ss.count) * sizeof(float),
                         cudaMemcpyDeviceToDevice, s.stream));
      P.drow_norm_max = ss.drow_norm_max;
      if (make_tc_rows(s, P.drows, ss.count, pq.view.dim, P.drows_tc, P.drows_map) != AEE_SUCCESS)
        return AEE_EFAILED;
    }
  }
  CK(cudaStreamSynchronize(s.stream));
  return AEE_SUCCESS;
}

// Validates a plan request and fills everything but the configuration.
AEEResult plan_setup(State& s, PqPlanImpl& P, const RoverSearchParams* p, int32_t nq, const int32_t* pool_sizes,
                     const int32_t* top_ks) {
  PqDevice& pq = s.pq;
  if (!pq.loaded || !pq.has_graph) { set_error("no PQ index with a graph is loaded"); return AEE_EFAILED; }
  if (!valid_params(p) || nq <= 0 || nq > kPlanMaxQueries || !pool_sizes) {
    set_error("plan: invalid parameters or query count (1..%d)", kPlanMaxQueries);
    return AEE_EBADPARM;
  }
  P.p = *p;
  P.nq = nq;
  P.epoch = pq.epoch;
  P.h_pool.assign(pool_sizes, pool_sizes + nq);
  P.max_pool = 0;
  for (int32_t v : P.h_pool) {
    if (v <= 0 || v > 4096) { set_error("pool sizes must be in 1..4096"); return AEE_EBADPARM; }
    P.max_pool = std::max(P.max_pool, v);
  }
  P.has_topk = top_ks != nullptr;
  P.max_k = p->top_k;
  if (top_ks) {
    P.max_k = 0;
    for (int i = 0; i < nq; ++i) P.max_k = std::max(P.max_k, top_ks[i]);
  }
  if (p->correction && pq.view.residual_bits == 0) { set_error("correction needs residuals"); return AEE_EBADPARM; }
  if (p->refine_budget > 0 && pq.view.residual_bits == 0) { set_error("refine needs residuals"); return AEE_EBADPARM; }
  if (p->third_residual && (!pq.view.e4.qparams || p->refine_budget <= 0)) {
    set_error("third_residual needs a loaded ERROR4 artifact and a refine budget");
    return AEE_EBADPARM;
  }
  P.expand = std::min(p->expand_count, pq.view.degree);
  if (P.expand > kMaxBatch) { set_error("expand_count above %d", kMaxBatch); return AEE_EBADPARM; }
  P.decodable = p->correction != 0 && pq.view.dim % 4 == 0;
  if (p->mode == ROVER_MODE_EXACT) {
    P.allow_packed = p->layout != ROVER_LAYOUT_DECODED;
    P.allow_decoded = P.decodable && p->layout != ROVER_LAYOUT_PACKED;
    if (p->layout == ROVER_LAYOUT_DECODED && !P.decodable) {
      set_error("the decoded layout needs correction on and dim %% 4 == 0");
      return AEE_EBADPARM;
    }
  } else if (p->mode == ROVER_MODE_BATCHED || p->mode == ROVER_MODE_GATED) {
    if (!P.decodable || p->layout == ROVER_LAYOUT_PACKED) {
      set_error("batched and gated plans need correction on, decoded rows and dim %% 4 == 0");
      return AEE_EBADPARM;
    }
    P.allow_decoded = true;
    P.gated = p->mode == ROVER_MODE_GATED && s.gate.enabled;
    P.W = p->beam_width;
    if (P.W == 0) P.W = std::max(1, std::min(kMaxBeamWidth, kMaxBatchIds / std::max(1, P.expand)));
    if (P.expand > 2 * 32 || P.W < 1 || P.W > kMaxBeamWidth || P.W * P.expand > kMaxBatchIds) {
      set_error("batched plan: need expand_count <= 64 and beam_width 1..%d with beam_width * expand_count <= %d",
                kMaxBeamWidth, kMaxBatchIds);
      return AEE_EBADPARM;
    }
  } else {
    set_error("unknown mode %d", p->mode);
    return AEE_EBADPARM;
  }
  if (P.allow_decoded) {
    bool ok = false;
    if (ensure_decoded(s, pq, &ok) != AEE_SUCCESS) return AEE_EFAILED;
    if (!ok) {
      if (!P.allow_packed) { set_error("decoded rows do not fit in device memory"); return AEE_ENOMEMORY; }
      P.allow_decoded = false;
    }
  }
  // widest beams first: each class is a contiguous run, and inside a class
  // the longest searches start first
  P.h_order.resize(nq);
  for (int i = 0; i < nq; ++i) P.h_order[i] = i;
  std::stable_sort(P.h_order.begin(), P.h_order.end(),
                   [&](int32_t x, int32_t y) { return P.h_pool[x] > P.h_pool[y]; });
  if (upload(P.pool, P.h_pool.data(), nq, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  if (upload(P.order, P.h_order.data(), nq, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  if (top_ks && upload(P.topk, top_ks, nq, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(P.ctl.ensure(sizeof(PlanControl)));
  PlanControl c0{};
  c0.gen = 1u;
  CK(cudaMemcpyAsync(P.ctl.p, &c0, sizeof(c0), cudaMemcpyHostToDevice, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  return plan_inputs(s, P);
}

}  // namespace

extern "C" AEEResult calculator_rover_pq_plan_create(remote_handle64 h, const RoverSearchParams* p, int32_t nq,
                                                     const int32_t* pool_sizes, const int32_t* top_ks,
                                                     const float* tune_queries, RoverPqPlan** plan) {
  (void)h;
  if (!plan) return AEE_EBADPARM;
  *plan = nullptr;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  auto* P = new (std::nothrow) PqPlanImpl();
  if (!P) return AEE_ENOMEMORY;
  auto fail = [&](AEEResult r) {
    P->release();
    P->magic = 0;
    delete P;
    return r;
  };
  AEEResult r = plan_setup(s, *P, p, nq, pool_sizes, top_ks);
  if (r != AEE_SUCCESS) return fail(r);
  PlanConfig def;
  def.layout = P->allow_decoded ? ROVER_LAYOUT_DECODED : ROVER_LAYOUT_PACKED;
  if (!tune_queries) {
    r = plan_configure(s, *P, def);
    if (r == AEE_EBADPARM) set_error("shared memory slices too large for pool %d", P->max_pool);
    if (r != AEE_SUCCESS) return fail(r);
    *plan = P;
    return AEE_SUCCESS;
  }
  if (P->allow_decoded && reinterpret_cast<uintptr_t>(tune_queries) % 16 != 0) {
    set_error("queries must be 16-byte aligned");
    return fail(AEE_EBADPARM);
  }
  // tuning outputs
  DevBuf ids, dists, counts, status;
  const int k = std::max(1, P->max_k);
  auto free_out = [&]() { ids.release(); dists.release(); counts.release(); status.release(); };
  if (ids.ensure(static_cast<size_t>(nq) * k * 4) != cudaSuccess ||
      dists.ensure(static_cast<size_t>(nq) * k * 4) != cudaSuccess || counts.ensure(static_cast<size_t>(nq) * 4) ||
      status.ensure(static_cast<size_t>(nq) * 4)) {
    free_out();
    set_error("out of device memory for the tuning outputs");
    return fail(AEE_ENOMEMORY);
  }
  RoverSearchOutputs o{};
  o.ids = ids.as<int32_t>();
  o.dists = dists.as<float>();
  o.counts = counts.as<int32_t>();
  o.out_stride = k;
  o.status = status.as<int32_t>();
  std::vector<PlanConfig> space;
  for (int layout : {ROVER_LAYOUT_DECODED, ROVER_LAYOUT_PACKED}) {
    if (layout == ROVER_LAYOUT_DECODED && !P->allow_decoded) continue;
    if (layout == ROVER_LAYOUT_PACKED && !P->allow_packed) continue;
    for (int split : {0, 1, 2}) {
      if (layout == ROVER_LAYOUT_PACKED) {
        PlanConfig c;
        c.layout = layout;
        c.split = split;
        space.push_back(c);
        continue;
      }
      for (int warps : {2, 4, 8})
        for (int vis : {1024, 2048, 4096}) {
          PlanConfig c;
          c.layout = layout;
          c.warps = warps;
          c.vis_cap = vis;
          c.split = split;
          space.push_back(c);
        }
    }
  }
  // the default first, so that its time is reported
  std::stable_sort(space.begin(), space.end(), [&](const PlanConfig& x, const PlanConfig& y) {
    const bool dx = x.layout == def.layout && x.warps == def.warps && x.vis_cap == def.vis_cap && x.split == 0;
    const bool dy = y.layout == def.layout && y.warps == def.warps && y.vis_cap == def.vis_cap && y.split == 0;
    return dx && !dy;
  });
  PlanConfig best;
  float best_ms = 0.0f;
  int tried = 0;
  for (const PlanConfig& c : space) {
    r = plan_configure(s, *P, c);
    if (r == AEE_EBADPARM) continue;   // slices do not fit
    if (r != AEE_SUCCESS) { free_out(); return fail(r); }
    float ms = 0.0f;
    bool overflow = false;
    for (int grow = 0; grow < 3; ++grow) {
      r = plan_time(s, *P, tune_queries, o, 2, &ms, &overflow);
      if (r != AEE_SUCCESS) { free_out(); return fail(r); }
      if (!overflow) break;
      P->table_scale *= 4;
      r = plan_configure(s, *P, c);
      if (r != AEE_SUCCESS) { free_out(); return fail(r == AEE_EBADPARM ? AEE_ENOMEMORY : r); }
    }
    if (overflow) continue;
    ++tried;
    if (tried == 1) P->default_ms = ms;
    if (best_ms == 0.0f || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  free_out();
  if (tried == 0) {
    set_error("no plan configuration fits (pool %d)", P->max_pool);
    return fail(AEE_EBADPARM);
  }
  // keep the winner's tables only
  P->visited.release();
  r = plan_configure(s, *P, best);
  if (r != AEE_SUCCESS) return fail(r);
  P->candidates = tried;
  P->tuned_ms = best_ms;
  *plan = P;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_pq_plan_create_fixed(remote_handle64 h, const RoverSearchParams* p,
                                                           int32_t nq, const int32_t* pool_sizes,
                                                           const int32_t* top_ks, const RoverPlanConfig* config,
                                                           RoverPqPlan** plan) {
  (void)h;
  if (!plan || !config) return AEE_EBADPARM;
  *plan = nullptr;
  const RoverPlanConfig& k = *config;
  const bool pow2 = k.shared_visited_slots >= 256 && k.shared_visited_slots <= 8192 &&
                    (k.shared_visited_slots & (k.shared_visited_slots - 1)) == 0;
  if ((k.layout != ROVER_LAYOUT_PACKED && k.layout != ROVER_LAYOUT_DECODED) || k.class_split < 0 ||
      k.class_split > 2 || (k.layout == ROVER_LAYOUT_DECODED && (!pow2 || k.warps_per_cta < 1 ||
                                                                 k.warps_per_cta > kMaxSearchWarps))) {
    set_error("plan configuration out of range");
    return AEE_EBADPARM;
  }
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  auto* P = new (std::nothrow) PqPlanImpl();
  if (!P) return AEE_ENOMEMORY;
  auto fail = [&](AEEResult r) {
    P->release();
    P->magic = 0;
    delete P;
    return r;
  };
  AEEResult r = plan_setup(s, *P, p, nq, pool_sizes, top_ks);
  if (r != AEE_SUCCESS) return fail(r);
  if ((k.layout == ROVER_LAYOUT_PACKED && !P->allow_packed) || (k.layout == ROVER_LAYOUT_DECODED && !P->allow_decoded)) {
    set_error("this request cannot run the %s layout", k.layout == ROVER_LAYOUT_PACKED ? "packed" : "decoded");
    return fail(AEE_EBADPARM);
  }
  PlanConfig c;
  c.layout = k.layout;
  c.warps = k.layout == ROVER_LAYOUT_PACKED ? kSearchWarps : k.warps_per_cta;
  c.vis_cap = k.layout == ROVER_LAYOUT_PACKED ? kSharedVisitedSlots : k.shared_visited_slots;
  c.split = k.class_split;
  r = plan_configure(s, *P, c);
  if (r == AEE_EBADPARM) set_error("shared memory slices too large for pool %d", P->max_pool);
  if (r != AEE_SUCCESS) return fail(r);
  *plan = P;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_pq_plan_launch(RoverPqPlan* plan, const float* queries,
                                                     const RoverSearchOutputs* out, void* stream) {
  PqPlanImpl* P = plan_cast(plan);
  if (!P || !queries || !out || !out->status || (out->ids && !out->counts)) return AEE_EBADPARM;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!s.pq.loaded || s.pq.epoch != P->epoch) {
    set_error("the index this plan was made on is no longer loaded");
    return AEE_EFAILED;
  }
  if (P->cfg.layout != ROVER_LAYOUT_PACKED && reinterpret_cast<uintptr_t>(queries) % 16 != 0) {
    set_error("queries must be 16-byte aligned");
    return AEE_EBADPARM;
  }
  cudaStream_t strm = stream ? static_cast<cudaStream_t>(stream) : s.stream;
  return plan_enqueue(s, *P, queries, *out, strm);
}

extern "C" AEEResult calculator_rover_pq_plan_describe(const RoverPqPlan* plan, RoverPlanInfo* info) {
  const PqPlanImpl* P = plan_cast(plan);
  if (!P || !info) return AEE_EBADPARM;
  RoverPlanInfo r{};
  r.num_queries = P->nq;
  r.mode = P->p.mode;
  r.layout = P->cfg.layout;
  r.warps_per_cta = P->cfg.warps;
  r.shared_visited_slots = P->cfg.layout == ROVER_LAYOUT_PACKED ? 0 : P->cfg.vis_cap;
  r.classes = static_cast<int32_t>(P->classes.size());
  const bool decoded = P->cfg.layout != ROVER_LAYOUT_PACKED;
  r.launches = 2 + (decoded ? 1 : 0) + ((decoded && (P->verify_seeds || P->gated)) ? 1 : 0) + r.classes;
  r.candidates = P->candidates;
  r.max_pool = P->max_pool;
  r.beam_width = P->p.mode == ROVER_MODE_EXACT ? 0 : P->W;
  for (int i = 0; i < r.classes && i < ROVER_PLAN_MAX_CLASSES; ++i) {
    r.class_pool[i] = P->classes[i].max_pool;
    r.class_queries[i] = P->classes[i].count;
    r.class_blocks[i] = P->classes[i].blocks;
  }
  r.tuned_ms = P->tuned_ms;
  r.default_ms = P->default_ms;
  r.device_bytes = static_cast<int64_t>(P->device_bytes());
  r.class_split = P->cfg.split;
  *info = r;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_pq_plan_destroy(RoverPqPlan* plan) {
  PqPlanImpl* P = plan_cast(plan);
  if (!P) return AEE_EBADPARM;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  P->release();
  P->magic = 0;
  delete P;
  return AEE_SUCCESS;
}

static_assert(sizeof(RoverGateTraceRow) == sizeof(GateTraceRow), "trace row layout");

extern "C" AEEResult calculator_rover_pq_trace(remote_handle64 h, const RoverSearchParams* p, const float* queries,
                                               int32_t nq, const int32_t* pool_sizes, const RoverSearchOutputs* out,
                                               RoverGateTraceRow* rows, int64_t capacity, int64_t* count) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!p || capacity < 0 || (capacity > 0 && !rows) || !count) return AEE_EBADPARM;
  CK(s.trace_rows.ensure(static_cast<size_t>(std::max<int64_t>(capacity, 1)) * sizeof(GateTraceRow)));
  CK(s.trace_count.ensure(sizeof(unsigned long long)));
  s.trace_dev = s.trace_rows.as<GateTraceRow>();
  s.trace_count_dev = s.trace_count.as<unsigned long long>();
  s.trace_cap = capacity;
  RoverSearchParams pp = *p;
  pp.mode = ROVER_MODE_BATCHED;
  pp.beam_width = 1;
  AEEResult r = pq_search_host(s, &pp, queries, nq, pool_sizes, nullptr, out);
  s.trace_dev = nullptr;
  s.trace_count_dev = nullptr;
  s.trace_cap = 0;
  if (r != AEE_SUCCESS) return r;
  unsigned long long n = 0;
  CK(cudaMemcpy(&n, s.trace_count.p, sizeof(n), cudaMemcpyDeviceToHost));
  *count = static_cast<int64_t>(n);
  const int64_t keep = std::min<int64_t>(capacity, static_cast<int64_t>(n));
  if (keep > 0) CK(cudaMemcpy(rows, s.trace_rows.p, static_cast<size_t>(keep) * sizeof(GateTraceRow),
                              cudaMemcpyDeviceToHost));
  return AEE_SUCCESS;
}

namespace {
uint16_t to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return static_cast<uint16_t>((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
  u += 0x7fffu + ((u >> 16) & 1u);
  return static_cast<uint16_t>(u >> 16);
}
}  // namespace

extern "C" AEEResult calculator_rover_gate_load(remote_handle64 h, const float* params, const float* mu,
                                                const float* sigma, const RoverGateThresholds* t) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!params || !mu || !sigma || !t) return AEE_EBADPARM;
  for (int i = 0; i < ROVER_GATE_PARAMS; ++i)
    if (!std::isfinite(params[i])) { set_error("gate parameter %d is not finite", i); return AEE_EBADPARM; }
  for (int i = 0; i < kGateIn; ++i)
    if (!std::isfinite(mu[i]) || !(sigma[i] > 0.0f) || !std::isfinite(sigma[i])) {
      set_error("gate input %d: mean / deviation invalid", i);
      return AEE_EBADPARM;
    }
  const float* w1 = params;                 // [5][64]
  const float* b1 = w1 + kGateIn * kGateHidden;
  const float* w2 = b1 + kGateHidden;       // [64][64]
  const float* b2 = w2 + kGateHidden * kGateHidden;
  const float* w3 = b2 + kGateHidden;       // [64][2]
  const float* b3 = w3 + kGateHidden * kGateOut;
  std::vector<uint16_t> w1t(kGateHidden * kGateW1Stride, 0), w2t(kGateHidden * kGateW2Stride, 0),
      w3t(8 * kGateW2Stride, 0);
  for (int o = 0; o < kGateHidden; ++o)
    for (int i = 0; i < kGateIn; ++i) w1t[o * kGateW1Stride + i] = to_bf16(w1[i * kGateHidden + o]);
  for (int o = 0; o < kGateHidden; ++o)
    for (int i = 0; i < kGateHidden; ++i) w2t[o * kGateW2Stride + i] = to_bf16(w2[i * kGateHidden + o]);
  for (int o = 0; o < kGateOut; ++o)
    for (int i = 0; i < kGateHidden; ++i) w3t[o * kGateW2Stride + i] = to_bf16(w3[i * kGateOut + o]);
  std::vector<float> bias(kGateHidden * 2 + 8, 0.0f);
  std::copy(b1, b1 + kGateHidden, bias.begin());
  std::copy(b2, b2 + kGateHidden, bias.begin() + kGateHidden);
  std::copy(b3, b3 + kGateOut, bias.begin() + 2 * kGateHidden);
  const size_t o1 = 0, o2 = o1 + w1t.size() * 2, o3 = o2 + w2t.size() * 2, ob = o3 + w3t.size() * 2;
  const size_t orow = (ob + bias.size() * 4 + 7) & ~static_cast<size_t>(7);   // MLP row counter
  const size_t total = orow + 8;
  CK(s.gate_buf.ensure(total));
  uint8_t* d = s.gate_buf.as<uint8_t>();
  CK(cudaMemcpy(d + o1, w1t.data(), w1t.size() * 2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + o2, w2t.data(), w2t.size() * 2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + o3, w3t.data(), w3t.size() * 2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + ob, bias.data(), bias.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemset(d + orow, 0, 8));
  GateParams g{};
  g.rows_evaluated = reinterpret_cast<unsigned long long*>(d + orow);
  g.w1t = reinterpret_cast<const uint16_t*>(d + o1);
  g.w2t = reinterpret_cast<const uint16_t*>(d + o2);
  g.w3t = reinterpret_cast<const uint16_t*>(d + o3);
  g.b1 = reinterpret_cast<const float*>(d + ob);
  g.b2 = g.b1 + kGateHidden;
  g.b3 = g.b2 + kGateHidden;
  for (int i = 0; i < kGateIn; ++i) {
    g.mu[i] = mu[i];
    g.inv_sigma[i] = 1.0f / sigma[i];
  }
  g.band_lo = t->band_lo;
  g.band_hi = t->band_hi;
  g.refine_logit = t->refine_logit;
  g.stop_logit = t->stop_logit;
  g.enabled = 1;
  s.gate = g;
  return AEE_SUCCESS;
}

namespace {
constexpr int kGateParamCount = ROVER_GATE_PARAMS;

// Device copies of one training set.
struct GateData {
  DevBuf x, y, m, mu, sigma, stats;
  AEEResult upload_rows(State& s, const float* hx, const float* hy, const float* hm, int64_t n) {
    if (upload(x, hx, static_cast<size_t>(n) * kGateIn, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
    if (upload(y, hy, static_cast<size_t>(n) * kGateOut, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
    if (upload(m, hm, static_cast<size_t>(n) * kGateOut, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
    return AEE_SUCCESS;
  }
  void release() { x.release(); y.release(); m.release(); mu.release(); sigma.release(); stats.release(); }
};
}  // namespace

extern "C" AEEResult calculator_rover_gate_grad(remote_handle64 h, const float* x, const float* y, const float* m,
                                                int64_t n, const float* params, const float* mu, const float* sigma,
                                                const float* pos_weight, float* grad_out, float* loss_out) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!x || !y || !m || n <= 0 || !params || !mu || !sigma || !pos_weight || !grad_out || !loss_out)
    return AEE_EBADPARM;
  GateData d;
  DevBuf p, g, l;
  AEEResult r = d.upload_rows(s, x, y, m, n);
  if (r == AEE_SUCCESS && (upload(p, params, kGateParamCount, s.stream) != AEE_SUCCESS ||
                           upload(d.mu, mu, kGateIn, s.stream) != AEE_SUCCESS ||
                           upload(d.sigma, sigma, kGateIn, s.stream) != AEE_SUCCESS))
    r = AEE_ENOMEMORY;
  if (r == AEE_SUCCESS) {
    if (g.ensure(kGateParamCount * sizeof(float)) != cudaSuccess || l.ensure(sizeof(double)) != cudaSuccess) {
      r = AEE_ENOMEMORY;
    } else {
      cudaMemsetAsync(g.p, 0, kGateParamCount * sizeof(float), s.stream);
      cudaMemsetAsync(l.p, 0, sizeof(double), s.stream);
      const cudaError_t e = launch_gate_fwd_bwd(p.as<float>(), d.mu.as<float>(), d.sigma.as<float>(), d.x.as<float>(),
                                                d.y.as<float>(), d.m.as<float>(), nullptr, n, pos_weight[0],
                                                pos_weight[1], static_cast<float>(n), g.as<float>(), l.as<double>(),
                                                s.stream);
      ++g_launches;
      double loss = 0.0;
      if (e != cudaSuccess ||
          cudaMemcpyAsync(grad_out, g.p, kGateParamCount * sizeof(float), cudaMemcpyDeviceToHost, s.stream) !=
              cudaSuccess ||
          cudaMemcpyAsync(&loss, l.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream) != cudaSuccess ||
          cudaStreamSynchronize(s.stream) != cudaSuccess) {
        set_error("gate gradient: %s", cudaGetErrorString(cudaGetLastError()));
        r = AEE_EFAILED;
      } else {
        *loss_out = static_cast<float>(loss / static_cast<double>(n));
      }
    }
  }
  d.release();
  p.release();
  g.release();
  l.release();
  return r;
}

extern "C" AEEResult calculator_rover_gate_train(remote_handle64 h, const float* x, const float* y, const float* m,
                                                 int64_t n, const RoverGateTrainParams* tp, float* params_out,
                                                 float* mu_out, float* sigma_out, float* epoch_loss) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!x || !y || !m || n <= 0 || !tp || tp->size < static_cast<int32_t>(offsetof(RoverGateTrainParams, reserved)) ||
      tp->epochs <= 0 || tp->batch <= 0 || !(tp->lr > 0.0f) || !params_out || !mu_out || !sigma_out)
    return AEE_EBADPARM;
  GateData d;
  DevBuf p, g, m1, m2, l, idx;
  auto fail = [&](AEEResult r) {
    d.release(); p.release(); g.release(); m1.release(); m2.release(); l.release(); idx.release();
    return r;
  };
  if (d.upload_rows(s, x, y, m, n) != AEE_SUCCESS) return fail(AEE_ENOMEMORY);
  // standardisation statistics
  if (d.stats.ensure(2 * kGateIn * sizeof(double)) != cudaSuccess) return fail(AEE_ENOMEMORY);
  cudaMemsetAsync(d.stats.p, 0, 2 * kGateIn * sizeof(double), s.stream);
  launch_gate_stats(d.x.as<float>(), n, d.stats.as<double>(), s.stream);
  ++g_launches;
  double acc[2 * kGateIn];
  if (cudaMemcpyAsync(acc, d.stats.p, sizeof(acc), cudaMemcpyDeviceToHost, s.stream) != cudaSuccess ||
      cudaStreamSynchronize(s.stream) != cudaSuccess) {
    set_error("gate statistics: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(AEE_EFAILED);
  }
  float mu[kGateIn], sigma[kGateIn];
  for (int i = 0; i < kGateIn; ++i) {
    const double mean = acc[i] / static_cast<double>(n);
    const double var = std::max(0.0, acc[kGateIn + i] / static_cast<double>(n) - mean * mean);
    mu[i] = static_cast<float>(mean);
    sigma[i] = static_cast<float>(std::max(std::sqrt(var), 1e-6));
  }
  if (upload(d.mu, mu, kGateIn, s.stream) != AEE_SUCCESS || upload(d.sigma, sigma, kGateIn, s.stream) != AEE_SUCCESS)
    return fail(AEE_ENOMEMORY);
  // He-uniform initialisation, zero biases
  std::vector<float> init(kGateParamCount, 0.0f);
  uint64_t rng = 0x9E3779B97F4A7C15ull ^ tp->seed;
  auto uni = [&rng]() {
    rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17;
    return static_cast<float>((rng >> 11) * (1.0 / 9007199254740992.0));
  };
  auto fill = [&](int off, int fan_in, int count) {
    const float lim = std::sqrt(6.0f / static_cast<float>(fan_in));
    for (int i = 0; i < count; ++i) init[off + i] = (2.0f * uni() - 1.0f) * lim;
  };
  fill(0, kGateIn, kGateIn * kGateHidden);
  fill(kGateIn * kGateHidden + kGateHidden, kGateHidden, kGateHidden * kGateHidden);
  fill(kGateIn * kGateHidden + kGateHidden + kGateHidden * kGateHidden + kGateHidden, kGateHidden,
       kGateHidden * kGateOut);
  if (upload(p, init.data(), init.size(), s.stream) != AEE_SUCCESS) return fail(AEE_ENOMEMORY);
  if (g.ensure(kGateParamCount * 4) != cudaSuccess || m1.ensure(kGateParamCount * 4) != cudaSuccess ||
      m2.ensure(kGateParamCount * 4) != cudaSuccess || l.ensure(sizeof(double)) != cudaSuccess ||
      idx.ensure(static_cast<size_t>(n) * sizeof(int64_t)) != cudaSuccess)
    return fail(AEE_ENOMEMORY);
  cudaMemsetAsync(m1.p, 0, kGateParamCount * 4, s.stream);
  cudaMemsetAsync(m2.p, 0, kGateParamCount * 4, s.stream);
  std::vector<int64_t> order(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) order[static_cast<size_t>(i)] = i;
  const float b1 = tp->beta1 > 0.f ? tp->beta1 : 0.9f, b2 = tp->beta2 > 0.f ? tp->beta2 : 0.999f;
  const float eps = tp->eps > 0.f ? tp->eps : 1e-8f;
  int64_t step = 0;
  for (int ep = 0; ep < tp->epochs; ++ep) {
    for (int64_t i = n - 1; i > 0; --i) {   // Fisher-Yates on the host, one upload per epoch
      const int64_t j = static_cast<int64_t>(uni() * static_cast<float>(i + 1)) % (i + 1);
      std::swap(order[static_cast<size_t>(i)], order[static_cast<size_t>(j)]);
    }
    if (cudaMemcpyAsync(idx.p, order.data(), order.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s.stream) !=
        cudaSuccess)
      return fail(AEE_EFAILED);
    cudaMemsetAsync(l.p, 0, sizeof(double), s.stream);
    for (int64_t b0 = 0; b0 < n; b0 += tp->batch) {
      const int64_t nb = std::min<int64_t>(tp->batch, n - b0);
      cudaMemsetAsync(g.p, 0, kGateParamCount * 4, s.stream);
      const cudaError_t e = launch_gate_fwd_bwd(p.as<float>(), d.mu.as<float>(), d.sigma.as<float>(), d.x.as<float>(),
                                                d.y.as<float>(), d.m.as<float>(), idx.as<int64_t>() + b0, nb,
                                                tp->pos_weight[0] > 0.f ? tp->pos_weight[0] : 1.0f,
                                                tp->pos_weight[1] > 0.f ? tp->pos_weight[1] : 1.0f,
                                                static_cast<float>(nb), g.as<float>(), l.as<double>(), s.stream);
      if (e != cudaSuccess) { set_error("gate training: %s", cudaGetErrorString(e)); return fail(AEE_EFAILED); }
      ++step;
      const float bc1 = 1.0f - std::pow(b1, static_cast<float>(step));
      const float bc2 = 1.0f - std::pow(b2, static_cast<float>(step));
      launch_gate_adam(p.as<float>(), g.as<float>(), m1.as<float>(), m2.as<float>(), kGateParamCount, tp->lr, b1, b2,
                       eps, tp->weight_decay, bc1, bc2, s.stream);
      g_launches += 2;
    }
    double loss = 0.0;
    if (cudaMemcpyAsync(&loss, l.p, sizeof(double), cudaMemcpyDeviceToHost, s.stream) != cudaSuccess ||
        cudaStreamSynchronize(s.stream) != cudaSuccess) {
      set_error("gate training: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(AEE_EFAILED);
    }
    if (epoch_loss) epoch_loss[ep] = static_cast<float>(loss / static_cast<double>(n));
  }
  if (cudaMemcpy(params_out, p.p, kGateParamCount * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return fail(AEE_EFAILED);
  std::copy(mu, mu + kGateIn, mu_out);
  std::copy(sigma, sigma + kGateIn, sigma_out);
  return fail(AEE_SUCCESS);
}

extern "C" AEEResult calculator_rover_seed_rank(remote_handle64 h, const float* queries, int32_t nq,
                                                const float* rows, int32_t n_rows, int32_t dim, float* out) {
  (void)h;
  if (!queries || !rows || !out || nq <= 0 || n_rows <= 0 || dim <= 0 || dim % 4 != 0 || dim > 1024)
    return AEE_EBADPARM;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  struct Bufs {
    DevBuf q, x, xtc, xn, o;
    ~Bufs() { q.release(); x.release(); xtc.release(); xn.release(); o.release(); }
  } b;
  if (upload(b.q, queries, static_cast<size_t>(nq) * dim, s.stream) ||
      upload(b.x, rows, static_cast<size_t>(n_rows) * dim, s.stream))
    return AEE_ENOMEMORY;
  CK(b.xn.ensure(static_cast<size_t>(n_rows) * sizeof(float)));
  CK(b.o.ensure(static_cast<size_t>(nq) * n_rows * sizeof(float)));
  launch_row_norms(b.x.as<float>(), n_rows, dim, b.xn.as<float>(), s.stream);
  CK(cudaGetLastError());
  ++g_launches;
  TcSeedMap map{};
  if (make_tc_rows(s, b.x, n_rows, dim, b.xtc, map) != AEE_SUCCESS) return AEE_EFAILED;
  if (seed_rank(s, b.q.as<float>(), 0, nq, dim, map, b.xtc.p ? b.xtc : b.x, b.xn, n_rows, b.o.as<float>(), n_rows,
                s.stream) != AEE_SUCCESS)
    return AEE_EFAILED;
  ++g_launches;
  CK(cudaMemcpyAsync(out, b.o.p, static_cast<size_t>(nq) * n_rows * sizeof(float), cudaMemcpyDeviceToHost, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  return check_tc_err(s);
}

extern "C" AEEResult calculator_rover_gate_rows(remote_handle64 h, uint64_t* rows) {
  (void)h;
  if (!rows) return AEE_EBADPARM;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  *rows = 0;
  if (!s.gate.enabled || !s.gate.rows_evaluated) return AEE_SUCCESS;
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  unsigned long long v = 0;
  CK(cudaMemcpy(&v, s.gate.rows_evaluated, sizeof(v), cudaMemcpyDeviceToHost));
  *rows = static_cast<uint64_t>(v);
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_gate_unload(remote_handle64 h) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  s.gate = GateParams{};
  s.gate_buf.release();
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_gate_eval(remote_handle64 h, const float* rows, int64_t n, float* logits) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (n < 0 || (n > 0 && (!rows || !logits))) return AEE_EBADPARM;
  if (!s.gate.enabled) { set_error("no gate loaded"); return AEE_EFAILED; }
  if (n == 0) return AEE_SUCCESS;
  DevBuf in, out;
  auto done = [&](AEEResult r) { in.release(); out.release(); return r; };
  if (in.ensure(static_cast<size_t>(n) * 5 * sizeof(float)) != cudaSuccess ||
      out.ensure(static_cast<size_t>(n) * 2 * sizeof(float)) != cudaSuccess) {
    set_error("out of device memory for %lld gate rows", static_cast<long long>(n));
    return done(AEE_ENOMEMORY);
  }
  if (cudaMemcpyAsync(in.p, rows, static_cast<size_t>(n) * 5 * sizeof(float), cudaMemcpyHostToDevice, s.stream) !=
      cudaSuccess)
    return done(AEE_EFAILED);
  launch_gate_eval(s.gate, in.as<float>(), n, out.as<float>(), s.stream);
  ++g_launches;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(logits, out.p, static_cast<size_t>(n) * 2 * sizeof(float), cudaMemcpyDeviceToHost,
                      s.stream) != cudaSuccess ||
      cudaStreamSynchronize(s.stream) != cudaSuccess) {
    set_error("gate evaluation failed: %s", cudaGetErrorString(cudaGetLastError()));
    return done(AEE_EFAILED);
  }
  return done(AEE_SUCCESS);
}

extern "C" AEEResult calculator_rover_seed_topm(remote_handle64 h, const float* rank, int32_t rows, int32_t n_seeds,
                                                int32_t m, uint64_t* keys, float* next) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (rows < 0 || n_seeds < 0 || m < 0 || (rows > 0 && (!rank || !next || (m > 0 && !keys)))) return AEE_EBADPARM;
  if (rows == 0 || m == 0) return AEE_SUCCESS;
  const size_t nr = static_cast<size_t>(rows) * n_seeds, nk = static_cast<size_t>(rows) * m;
  DevBuf in, out_keys, out_next;
  auto done = [&](AEEResult r) { in.release(); out_keys.release(); out_next.release(); return r; };
  if (in.ensure(std::max<size_t>(nr, 1) * sizeof(float)) != cudaSuccess ||
      out_keys.ensure(nk * sizeof(uint64_t)) != cudaSuccess ||
      out_next.ensure(static_cast<size_t>(rows) * sizeof(float)) != cudaSuccess) {
    set_error("out of device memory for %d x %d ranks", rows, n_seeds);
    return done(AEE_ENOMEMORY);
  }
  if (nr && cudaMemcpyAsync(in.p, rank, nr * sizeof(float), cudaMemcpyHostToDevice, s.stream) != cudaSuccess)
    return done(AEE_EFAILED);
  launch_pq_seed_topm(in.as<float>(), n_seeds, n_seeds, rows, m, out_keys.as<uint64_t>(), out_next.as<float>(),
                      s.stream);
  ++g_launches;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(keys, out_keys.p, nk * sizeof(uint64_t), cudaMemcpyDeviceToHost, s.stream) != cudaSuccess ||
      cudaMemcpyAsync(next, out_next.p, static_cast<size_t>(rows) * sizeof(float), cudaMemcpyDeviceToHost,
                      s.stream) != cudaSuccess ||
      cudaStreamSynchronize(s.stream) != cudaSuccess) {
    set_error("seed selection failed: %s", cudaGetErrorString(cudaGetLastError()));
    return done(AEE_EFAILED);
  }
  return done(AEE_SUCCESS);
}

extern "C" AEEResult calculator_rover_pq_lut(remote_handle64 h, const float* queries, int32_t nq, float* out_luts,
                                             int32_t* out_status) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!s.pq.loaded) { set_error("no PQ index loaded"); return AEE_EFAILED; }
  if (nq <= 0 || !queries || !out_luts) return AEE_EBADPARM;
  const PqIndexView& v = s.pq.view;
  const size_t lut = static_cast<size_t>(v.m) * v.ks;
  if (upload(s.in_queries, queries, static_cast<size_t>(nq) * v.dim, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(s.luts.ensure(nq * lut * 4));
  CK(s.status.ensure(nq * 4));
  CK(cudaMemsetAsync(s.status.p, 0, nq * 4, s.stream));
  launch_pq_lut(v, s.in_queries.as<float>(), nq, s.luts.as<float>(), s.status.as<int32_t>(), s.stream);
  CK(cudaGetLastError());
  ++g_launches;
  std::vector<int32_t> hs(nq);
  if (download(out_luts, s.luts.p, nq * lut, s.stream) || download(hs.data(), s.status.p, nq, s.stream)) return AEE_EFAILED;
  CK(cudaStreamSynchronize(s.stream));
  if (out_status) std::copy(hs.begin(), hs.end(), out_status);
  for (int32_t x : hs) if (x) return AEE_EFAILED;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_score(remote_handle64 h, int32_t kind, const float* queries, int32_t nq,
                                            const int32_t* ids, const int64_t* offsets, float* out_dists,
                                            int32_t* out_status) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (nq <= 0 || !queries || !offsets || !out_dists || kind < 0 || kind > 4) return AEE_EBADPARM;
  const bool pqk = kind <= 1 || kind == 4;
  if (pqk && !s.pq.loaded) { set_error("no PQ index loaded"); return AEE_EFAILED; }
  if (!pqk && !s.sq.loaded) { set_error("no SQ index loaded"); return AEE_EFAILED; }
  if ((kind == 1 || kind == 4) && !s.pq.view.residual_bits) return AEE_EBADPARM;
  if (kind == 4) {
    bool ok = false;
    if (s.pq.view.dim % 4 != 0 || s.pq.view.dim > 384) {
      set_error("kind 4 needs dim %% 4 == 0 and dim <= 384 (its 32-row tiles live in shared memory)");
      return AEE_EBADPARM;
    }
    if (ensure_decoded(s, s.pq, &ok) != AEE_SUCCESS) return AEE_EFAILED;
    if (!ok) { set_error("decoded rows do not fit in device memory"); return AEE_ENOMEMORY; }
  }
  const int dim = pqk ? s.pq.view.dim : s.sq.view.dim;
  const int64_t total = offsets[nq];
  for (int i = 0; i < nq; ++i)
    if (offsets[i + 1] < offsets[i] || offsets[0] != 0) return AEE_EBADPARM;
  if (upload(s.in_queries, queries, static_cast<size_t>(nq) * dim, s.stream) ||
      upload(s.in_offsets, offsets, nq + 1, s.stream) || upload(s.in_ids, ids, static_cast<size_t>(total), s.stream))
    return AEE_ENOMEMORY;
  CK(s.out_dists.ensure(std::max<int64_t>(total, 1) * 4));
  CK(s.status.ensure(nq * 4));
  CK(cudaMemsetAsync(s.status.p, 0, nq * 4, s.stream));
  const int32_t* di = s.in_ids.as<int32_t>();
  const int64_t* dof = s.in_offsets.as<int64_t>();
  float* dout = s.out_dists.as<float>();
  int32_t* dst = s.status.as<int32_t>();
  if (kind == 0) {
    const size_t lut = static_cast<size_t>(s.pq.view.m) * s.pq.view.ks;
    CK(s.luts.ensure(nq * lut * 4));
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_LUT, s.stream);
      launch_pq_lut(s.pq.view, s.in_queries.as<float>(), nq, s.luts.as<float>(), dst, s.stream);
    }
    TimedLaunch tl(ROVER_KERNEL_PQ_ADC, s.stream);
    launch_pq_adc(s.pq.view, s.luts.as<float>(), nq, di, dof, dout, dst, s.stream);
    ++g_launches;
  } else if (kind == 1) {
    TimedLaunch tl(ROVER_KERNEL_PQ_RESIDUAL, s.stream);
    launch_pq_residual(s.pq.view, s.in_queries.as<float>(), nq, di, dof, dout, dst, s.stream);
  } else if (kind == 2) {
    TimedLaunch tl(ROVER_KERNEL_SQ_COARSE, s.stream);
    launch_sq_coarse(s.sq.view, s.in_queries.as<float>(), nq, di, dof, dout, dst, s.stream);
  } else if (kind == 3) {
    TimedLaunch tl(ROVER_KERNEL_SQ_EXACT, s.stream);
    launch_sq_exact(s.sq.view, s.in_queries.as<float>(), nq, di, dof, dout, dst, s.stream);
  } else {
    TimedLaunch tl(ROVER_KERNEL_PQ_RESCORE, s.stream);
    launch_pq_rescore(s.pq.view.dim, s.pq.view.n, s.pq.decoded.as<float>(), s.in_queries.as<float>(), nq, di, dof,
                      dout, dst, s.stream);
  }
  CK(cudaGetLastError());
  ++g_launches;
  std::vector<int32_t> hs(nq);
  if (download(out_dists, dout, static_cast<size_t>(total), s.stream) || download(hs.data(), dst, nq, s.stream))
    return AEE_EFAILED;
  CK(cudaStreamSynchronize(s.stream));
  collect_timings();
  if (out_status) std::copy(hs.begin(), hs.end(), out_status);
  for (int32_t x : hs) if (x) { set_error("score failed with status %d", x); return AEE_EFAILED; }
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_refine(remote_handle64 h, int32_t kind, const float* queries, int32_t nq,
                                             const int32_t* cand_ids, int32_t cand_stride,
                                             const int32_t* cand_counts, int32_t top_k, int32_t* out_ids,
                                             float* out_dists, int32_t* out_counts, int32_t* out_status) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (nq <= 0 || !queries || !cand_ids || !cand_counts || top_k <= 0 || cand_stride <= 0 || kind < 0 || kind > 4)
    return AEE_EBADPARM;
  // kinds 3 / 4: kinds 0 / 1 in mode ERROR4 (the index's third-level term)
  const bool error4 = kind >= 3;
  if (error4) {
    kind -= 3;
    const Error4View& e = kind == 1 ? s.pq.view.e4 : s.sq.view.e4;
    if (!e.qparams) { set_error("no ERROR4 artifact is loaded for this index"); return AEE_EFAILED; }
  }
  if (kind == 1 && (!s.pq.loaded || !s.pq.view.residual_bits)) { set_error("no PQ residual index"); return AEE_EFAILED; }
  if (kind == 0 && (!s.sq.loaded || !s.sq.view.residual)) { set_error("no SQ residual index"); return AEE_EFAILED; }
  if (kind == 2 && !s.sq.loaded) { set_error("no SQ index loaded"); return AEE_EFAILED; }
  const int dim = kind == 1 ? s.pq.view.dim : s.sq.view.dim;
  int cap = 1;
  for (int i = 0; i < nq; ++i) {
    if (cand_counts[i] < 0 || cand_counts[i] > cand_stride || cand_counts[i] > 2048) return AEE_EBADPARM;
    cap = std::max(cap, cand_counts[i]);
  }
  if (upload(s.in_queries, queries, static_cast<size_t>(nq) * dim, s.stream) ||
      upload(s.in_ids, cand_ids, static_cast<size_t>(nq) * cand_stride, s.stream) ||
      upload(s.in_pool, cand_counts, nq, s.stream))
    return AEE_ENOMEMORY;
  CK(s.out_ids.ensure(static_cast<size_t>(nq) * top_k * 4));
  CK(s.out_dists.ensure(static_cast<size_t>(nq) * top_k * 4));
  CK(s.out_counts.ensure(nq * 4));
  CK(s.status.ensure(nq * 4));
  CK(cudaMemsetAsync(s.status.p, 0, nq * 4, s.stream));
  // PQ: read the decode from the decoded rows when they are (or can be) built
  const float* decoded = nullptr;
  if (kind == 1 && s.pq.view.dim % 4 == 0) {
    bool ok = false;
    if (ensure_decoded(s, s.pq, &ok) != AEE_SUCCESS) return AEE_EFAILED;
    if (ok) decoded = s.pq.decoded.as<float>();
  }
  if (kind == 2) {
    TimedLaunch tl(ROVER_KERNEL_REFINE, s.stream);
    launch_rerank(s.sq.view, s.in_queries.as<float>(), nq, s.in_ids.as<int32_t>(), cand_stride,
                  s.in_pool.as<int32_t>(), top_k, cap, s.out_ids.as<int32_t>(), s.out_dists.as<float>(),
                  s.out_counts.as<int32_t>(), s.status.as<int32_t>(), s.stream);
  } else {
    TimedLaunch tl(ROVER_KERNEL_REFINE, s.stream);
    launch_refine(kind, s.pq.view, s.sq.view, decoded, s.in_queries.as<float>(), nq, s.in_ids.as<int32_t>(), cand_stride,
                  s.in_pool.as<int32_t>(), top_k, cap, s.out_ids.as<int32_t>(), s.out_dists.as<float>(),
                  s.out_counts.as<int32_t>(), s.status.as<int32_t>(), s.stream, error4);
  }
  CK(cudaGetLastError());
  ++g_launches;
  ResultStage rs(s);
  rs.add(out_ids, s.out_ids.p, static_cast<size_t>(nq) * top_k * sizeof(int32_t));
  rs.add(out_dists, s.out_dists.p, static_cast<size_t>(nq) * top_k * sizeof(float));
  rs.add(out_counts, s.out_counts.p, static_cast<size_t>(nq) * sizeof(int32_t));
  if (rs.arm() != AEE_SUCCESS) return AEE_ENOMEMORY;
  if (fetch_status(s, s.status.as<int32_t>(), nq, s.stream) != AEE_SUCCESS) return AEE_EFAILED;
  collect_timings();
  if (rs.finish(s.stream) != AEE_SUCCESS) return AEE_EFAILED;
  if (out_status) std::copy(s.h_status.begin(), s.h_status.begin() + nq, out_status);
  for (int i = 0; i < nq; ++i)
    if (s.h_status[i]) { set_error("refine failed with status %d", s.h_status[i]); return AEE_EFAILED; }
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_sq_load(remote_handle64 h, const RoverSqIndexDesc* desc) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!desc) return AEE_EBADPARM;
  return load_sq(s, s.sq, desc, desc->l1_bits);
}

extern "C" AEEResult calculator_rover_sq_unload(remote_handle64 h) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  s.sq.release();
  return AEE_SUCCESS;
}

// retrieval_pq_train (retrieval_pq_core.c:202-224) on the device.
extern "C" AEEResult calculator_rover_pq_train(remote_handle64 h, const float* train_vectors, int32_t train_count,
                                               int32_t dim, int32_t m, int32_t ks, int32_t kmeans_iters,
                                               float* out_codebook) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  // retrieval_pq_validate_config (:84-93) and the input checks of :108-129
  if (!train_vectors || !out_codebook || train_count <= 0 || m <= 0 || ks <= 0 || ks > 256 || dim <= 0 ||
      dim % m != 0)
    return AEE_EBADPARM;
  const size_t values = static_cast<size_t>(train_count) * dim;
  for (size_t i = 0; i < values; ++i)
    if (!std::isfinite(train_vectors[i])) { set_error("training vector %zu is not finite", i / dim); return AEE_EBADPARM; }
  DevBuf x, book;
  const size_t book_floats = static_cast<size_t>(ks) * dim;   // m * ks * subdim
  if (upload(x, train_vectors, values, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(book.ensure(book_floats * sizeof(float)));
  PqTrainScratch scratch;
  {
    TimedLaunch tl(ROVER_KERNEL_PQ_TRAIN, s.stream);
    CK(pq_train_device(x.as<float>(), train_count, dim, m, ks, kmeans_iters, book.as<float>(), &scratch, s.stream));
  }
  g_launches += static_cast<unsigned long long>(pq_train_launches(kmeans_iters));
  if (download(out_codebook, book.p, book_floats, s.stream)) return AEE_EFAILED;
  CK(cudaStreamSynchronize(s.stream));
  return AEE_SUCCESS;
}

// retrieval_pq_encode_batch (retrieval_pq_core.c:226-268) on the device, in
// chunks of at most 1M vectors.
extern "C" AEEResult calculator_rover_pq_encode(remote_handle64 h, const float* vectors, int64_t count, int32_t dim,
                                                const float* codebook, int32_t m, int32_t ks, uint8_t* out_codes) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!vectors || !codebook || !out_codes || count < 0 || m <= 0 || ks <= 0 || ks > 256 || dim <= 0 ||
      dim % m != 0)
    return AEE_EBADPARM;
  if (count == 0) return AEE_SUCCESS;
  const int code_bytes = ks <= 16 ? m / 2 + m % 2 : m;
  DevBuf book, x, codes, bad;
  if (upload(book, codebook, static_cast<size_t>(ks) * dim, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(bad.ensure(sizeof(int)));
  CK(cudaMemsetAsync(bad.p, 0, sizeof(int), s.stream));
  const int64_t chunk = 1 << 20;
  for (int64_t begin = 0; begin < count; begin += chunk) {
    const int64_t nc = std::min<int64_t>(chunk, count - begin);
    if (upload(x, vectors + begin * dim, static_cast<size_t>(nc) * dim, s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
    CK(codes.ensure(static_cast<size_t>(nc) * code_bytes));
    {
      TimedLaunch tl(ROVER_KERNEL_PQ_TRAIN, s.stream);
      launch_pq_encode(x.as<float>(), nc, dim, m, ks, book.as<float>(), codes.as<uint8_t>(), bad.as<int>(), s.stream);
    }
    CK(cudaGetLastError());
    ++g_launches;
    if (download(out_codes + begin * code_bytes, codes.p, static_cast<size_t>(nc) * code_bytes, s.stream))
      return AEE_EFAILED;
  }
  int h_bad = 0;
  CK(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  if (h_bad) { set_error("a subspace distance is not finite"); return AEE_EBADPARM; }
  return AEE_SUCCESS;
}

// The ERROR4 payload of retrieval_final_refine's mode 2 (the host validated
// the artifact's header, retrieval_final_refine.c:118-166; the qparams
// checks of :160-163 are repeated here).
extern "C" AEEResult calculator_rover_error4_load(remote_handle64 h, int32_t kind, const float* qparams,
                                                  const uint8_t* code_blocks, int64_t code_blocks_bytes,
                                                  int32_t num_vectors, int32_t dim) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if ((kind != 0 && kind != 1) || !qparams || !code_blocks || num_vectors <= 0 || dim <= 0 || dim > 8192)
    return AEE_EBADPARM;
  const bool pq = kind == 1;
  if (pq ? !s.pq.loaded : !s.sq.loaded) { set_error("no index of this kind is loaded"); return AEE_EFAILED; }
  if (pq ? session_busy(s, kSessionPurePq) : session_busy(s, kSessionSqmd)) return AEE_EFAILED;
  const int32_t n = pq ? s.pq.view.n : s.sq.view.n;
  const int32_t idim = pq ? s.pq.view.dim : s.sq.view.dim;
  const int cb = (dim + 1) / 2, vpb = 4096 / cb;
  if (num_vectors != n || dim != idim || vpb <= 0 ||
      code_blocks_bytes != static_cast<int64_t>((num_vectors + vpb - 1) / vpb) * 4096) {
    set_error("ERROR4 artifact does not match the loaded index");
    return AEE_EBADPARM;
  }
  for (int64_t i = 0; i < num_vectors; ++i)
    if (!std::isfinite(qparams[2 * i]) || qparams[2 * i] < 0.0f || !std::isfinite(qparams[2 * i + 1])) {
      set_error("ERROR4 qparams of row %lld are invalid", static_cast<long long>(i));
      return AEE_EBADPARM;
    }
  DevBuf& q = pq ? s.pq.e4_qparams : s.sq.e4_qparams;
  DevBuf& b = pq ? s.pq.e4_blocks : s.sq.e4_blocks;
  if (upload(q, qparams, static_cast<size_t>(num_vectors) * 2, s.stream) != AEE_SUCCESS ||
      upload(b, code_blocks, static_cast<size_t>(code_blocks_bytes), s.stream) != AEE_SUCCESS)
    return AEE_ENOMEMORY;
  CK(cudaStreamSynchronize(s.stream));
  Error4View& e = pq ? s.pq.view.e4 : s.sq.view.e4;
  e.qparams = q.as<float>();
  e.blocks = b.as<uint8_t>();
  e.code_bytes = cb;
  e.vpb = vpb;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_error4_unload(remote_handle64 h, int32_t kind) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (kind != 0 && kind != 1) return AEE_EBADPARM;
  if (kind == 1) {
    s.pq.e4_qparams.release(); s.pq.e4_blocks.release(); s.pq.view.e4 = Error4View{};
  } else {
    s.sq.e4_qparams.release(); s.sq.e4_blocks.release(); s.sq.view.e4 = Error4View{};
  }
  return AEE_SUCCESS;
}

// The SQMD split-distance bias (sqmd_load_correction_bias,
// retrieval_rpc_demo_support.c:237-297; the host checked the header and the
// payload hash).  Split distance needs 4-bit L1 codes and residuals
// (sqmd_split_query_init, retrieval_rpc_demo_pipeline.c:916-933).
extern "C" AEEResult calculator_rover_sq_split_load(remote_handle64 h, const float* bias, int32_t num_vectors) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!bias || num_vectors <= 0) return AEE_EBADPARM;
  SqDevice& d = s.sq;
  if (!d.loaded || num_vectors != d.view.n) { set_error("the bias does not match the loaded SQ index"); return AEE_EBADPARM; }
  if (d.view.l1_bits != 4 || !d.view.residual || !d.view.qparams || !std::isfinite(d.view.l1_scale) ||
      !(d.view.l1_scale > 0.0f) || !std::isfinite(d.view.l1_zero)) {
    set_error("split distance needs 4-bit L1 codes, residuals and a valid L1 scale");
    return AEE_EBADPARM;
  }
  for (int32_t i = 0; i < num_vectors; ++i)
    if (!std::isfinite(bias[i])) { set_error("bias of row %d is not finite", i); return AEE_EBADPARM; }
  if (upload(d.split_bias, bias, static_cast<size_t>(num_vectors), s.stream) != AEE_SUCCESS) return AEE_ENOMEMORY;
  CK(cudaStreamSynchronize(s.stream));
  d.view.split_bias = d.split_bias.as<float>();
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_sq_search(remote_handle64 h, const RoverSearchParams* p, const float* queries,
                                                int32_t nq, const int32_t* pool_sizes, const RoverSearchOutputs* out) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (!valid_params(p) || nq < 0 || !out || !out->ids || !out->dists || !out->counts || out->out_stride <= 0 ||
      !queries || !pool_sizes)
    return AEE_EBADPARM;
  if (nq == 0) return AEE_SUCCESS;
  if (!s.sq.loaded || !s.sq.view.graph) { set_error("no SQ index with a graph loaded"); return AEE_EFAILED; }
  if (p->sq_mode < 0 || p->sq_mode > 2) { set_error("sq_mode must be 0, 1 or 2"); return AEE_EBADPARM; }
  if (p->sq_mode != 0 && p->correction && !s.sq.view.residual) {
    set_error("correction needs residuals");
    return AEE_EBADPARM;
  }
  if (p->split_distance && (p->sq_mode != 1 || !p->correction || !s.sq.view.split_bias)) {
    set_error("split_distance needs sq_mode 1, correction and a loaded split bias");
    return AEE_EBADPARM;
  }
  const int dim = s.sq.view.dim;
  std::vector<int32_t> h_pool(pool_sizes, pool_sizes + nq);
  const int stride = out->out_stride;
  if (upload(s.in_queries, queries, static_cast<size_t>(nq) * dim, s.stream) ||
      upload(s.in_pool, pool_sizes, nq, s.stream))
    return AEE_ENOMEMORY;
  CK(s.out_ids.ensure(static_cast<size_t>(nq) * stride * 4));
  CK(s.out_dists.ensure(static_cast<size_t>(nq) * stride * 4));
  CK(s.out_counts.ensure(nq * 4));
  CK(s.stats.ensure(static_cast<size_t>(nq) * 32));
  CK(s.status.ensure(nq * 4));
  const int mode = p->sq_mode == 1 ? kSqModeSqmd : p->sq_mode == 2 ? kSqModeDb : kSqModeDsp;
  ResultStage rs(s);
  rs.add(out->ids, s.out_ids.p, static_cast<size_t>(nq) * stride * sizeof(int32_t));
  rs.add(out->dists, s.out_dists.p, static_cast<size_t>(nq) * stride * sizeof(float));
  rs.add(out->counts, s.out_counts.p, static_cast<size_t>(nq) * sizeof(int32_t));
  if (out->stats) rs.add(out->stats, s.stats.p, static_cast<size_t>(nq) * 4 * sizeof(uint64_t));
  if (rs.arm() != AEE_SUCCESS) return AEE_ENOMEMORY;
  AEEResult r = sq_search_core(s, s.sq, mode, p, s.in_queries.as<float>(), nq,
                               s.in_pool.as<int32_t>(), h_pool, p->sq_mode == 1 ? stride : std::min(stride, p->top_k),
                               s.out_ids.as<int32_t>(), s.out_dists.as<float>(), stride, s.out_counts.as<int32_t>(),
                               s.stats.as<unsigned long long>(), s.status.as<int32_t>(), s.stream);
  if (out->status) std::copy(s.h_status.begin(), s.h_status.begin() + nq, out->status);
  if (r != AEE_SUCCESS) return r;
  return rs.finish(s.stream);
}

// ===========================================================================
// Reference interface (include/calculator.h)

extern "C" int calculator_open(const char* uri, remote_handle64* handle) {
  (void)uri;
  if (!handle) return AEE_EBADPARM;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  ++open_count;
  *handle = static_cast<remote_handle64>(open_count);
  return AEE_SUCCESS;
}

extern "C" int calculator_close(remote_handle64 handle) {
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (handle && open_count > 0) --open_count;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_rover_configure(remote_handle64 h, int32 abi_version, int32 l1_bits) {
  (void)h;
  if (abi_version != 1 || (l1_bits != 4 && l1_bits != 8)) return AEE_EBADPARM;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  s.l1_bits = l1_bits;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_retrieval_load(remote_handle64 h, const int* graph, int graphLen, const uint8* l1_codes,
                                               int l1_codesLen, int32 num_vectors, int32 dim, int32 graph_k,
                                               int32 graph_entry_point, float l1_scale, float l1_zero_point) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (session_busy(s, kSessionSqmd)) return AEE_EFAILED;
  s.legacy.release();
  s.legacy_dma = false;
  if (num_vectors <= 0 || dim <= 0 || graph_k <= 0 || dim > 1024) return AEE_EBADPARM;
  const int cb = s.l1_bits == 4 ? (dim + 1) / 2 : dim;
  if (graphLen < static_cast<int64_t>(num_vectors) * graph_k || l1_codesLen < static_cast<int64_t>(num_vectors) * cb)
    return AEE_EBADPARM;
  RoverSqIndexDesc d{};
  d.graph = graph;
  d.num_vectors = num_vectors;
  d.graph_degree = graph_k;
  d.graph_entry = (graph_entry_point >= 0 && graph_entry_point < num_vectors) ? graph_entry_point : -1;
  d.dim = dim;
  d.l1_codes = l1_codes;
  d.l1_scale = l1_scale;
  d.l1_zero = l1_zero_point;
  return load_sq(s, s.legacy, &d, s.l1_bits) == AEE_SUCCESS ? AEE_SUCCESS : AEE_ENOMEMORY;
}

extern "C" AEEResult calculator_retrieval_search(remote_handle64 h, const float* query, int queryLen,
                                                 int32 entry_points, int32 expand_count, int32 pool_size,
                                                 int32 num_out, int* candidate_ids, int candidate_idsLen,
                                                 float* candidate_dists, int candidate_distsLen,
                                                 int32* actual_count) {
  (void)h;
  if (!actual_count) return AEE_EBADPARM;
  *actual_count = 0;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (!s.legacy.loaded || !s.legacy.view.graph) return AEE_EFAILED;
  if (queryLen < s.legacy.view.dim || pool_size <= 0 || num_out <= 0) return AEE_EBADPARM;
  if (candidate_idsLen < num_out || candidate_distsLen < num_out) return AEE_EBADPARM;
  if (std::min(expand_count, s.legacy.view.degree) <= 0) return AEE_EBADPARM;
  // with no entry points the reference's loop seeds nothing and returns an
  // empty result (retrieval_async_dsp_search.c:438)
  if (entry_points <= 0) return AEE_SUCCESS;
  RoverSearchParams p{};
  p.size = sizeof(p);
  p.entry_points = entry_points;
  p.seed = 42u;
  p.expand_count = expand_count;
  const int pool = std::min(pool_size, 2000);
  std::vector<int32_t> h_pool(1, pool);
  if (upload(s.in_queries, query, s.legacy.view.dim, s.stream) || upload(s.in_pool, h_pool.data(), 1, s.stream))
    return AEE_ENOMEMORY;
  CK(s.out_ids.ensure(num_out * 4));
  CK(s.out_dists.ensure(num_out * 4));
  CK(s.out_counts.ensure(4));
  CK(s.status.ensure(4));
  AEEResult r = sq_search_core(s, s.legacy, kSqModeDsp, &p, s.in_queries.as<float>(), 1, s.in_pool.as<int32_t>(),
                               h_pool, num_out, s.out_ids.as<int32_t>(), s.out_dists.as<float>(), num_out,
                               s.out_counts.as<int32_t>(), nullptr, s.status.as<int32_t>(), s.stream);
  if (r != AEE_SUCCESS) return AEE_EFAILED;
  int32_t count = 0;
  if (download(&count, s.out_counts.p, 1, s.stream)) return AEE_EFAILED;
  CK(cudaStreamSynchronize(s.stream));
  if (download(candidate_ids, s.out_ids.p, count, s.stream) ||
      download(candidate_dists, s.out_dists.p, count, s.stream))
    return AEE_EFAILED;
  CK(cudaStreamSynchronize(s.stream));
  *actual_count = count;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_retrieval_unload(remote_handle64 h) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (session_busy(s, kSessionSqmd)) return AEE_EFAILED;
  s.legacy.release();
  s.legacy_dma = false;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_retrieval_load_dma(remote_handle64 h, int32 fd_graph, const int32* fd_l1_codes,
                                                   int fd_l1_codesLen, int32 l1_chunk_vectors, int32 num_vectors,
                                                   int32 dim, int32 graph_k, int32 graph_entry_point, float l1_scale,
                                                   float l1_zero_point) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;
  if (session_busy(s, kSessionSqmd)) return AEE_EFAILED;
  s.legacy.release();
  s.legacy_dma = false;
  if (fd_graph < -1 || num_vectors <= 0 || dim <= 0 || graph_k <= 0 || dim > 1024) return AEE_EBADPARM;
  if (!fd_l1_codes || fd_l1_codesLen < 1 || fd_l1_codesLen > 16 || l1_chunk_vectors <= 0) return AEE_EBADPARM;
  const int cb = s.l1_bits == 4 ? (dim + 1) / 2 : dim;
  std::vector<uint8_t> codes(static_cast<size_t>(num_vectors) * cb);
  size_t done = 0;
  for (int c = 0; c < fd_l1_codesLen; ++c) {
    void* ptr = nullptr;
    size_t bytes = 0;
    if (rover_rpcmem_lookup(fd_l1_codes[c], &ptr, &bytes) != 0) return AEE_EFAILED;
    const size_t want = std::min(static_cast<size_t>(l1_chunk_vectors) * cb, codes.size() - done);
    if (bytes < want) return AEE_EFAILED;
    std::memcpy(codes.data() + done, ptr, want);
    done += want;
  }
  if (done != codes.size()) return AEE_EBADPARM;
  RoverSqIndexDesc d{};
  void* gptr = nullptr;
  size_t gbytes = 0;
  if (fd_graph != -1) {
    if (rover_rpcmem_lookup(fd_graph, &gptr, &gbytes) != 0 ||
        gbytes < static_cast<size_t>(num_vectors) * graph_k * sizeof(int32_t))
      return AEE_EFAILED;
    d.graph = static_cast<const int32_t*>(gptr);
  }
  d.num_vectors = num_vectors;
  d.graph_degree = graph_k;
  d.graph_entry = (graph_entry_point >= 0 && graph_entry_point < num_vectors) ? graph_entry_point : -1;
  d.dim = dim;
  d.l1_codes = codes.data();
  d.l1_scale = l1_scale;
  d.l1_zero = l1_zero_point;
  if (load_sq(s, s.legacy, &d, s.l1_bits) != AEE_SUCCESS) return AEE_ENOMEMORY;
  s.legacy_dma = true;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_retrieval_unload_dma(remote_handle64 h) {
  (void)h;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (!s.legacy_dma) return AEE_SUCCESS;
  if (session_busy(s, kSessionSqmd)) return AEE_EFAILED;
  s.legacy.release();
  s.legacy_dma = false;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_retrieval_pure_pq_load_dma(
    remote_handle64 h, const int32* fd_pq_codes, int fd_pq_codesLen, const int32* pq_chunk_vector_counts,
    int pq_chunk_vector_countsLen, int32 pq_chunk_vectors, const float* pq_codebook, int pq_codebookLen,
    int32 num_vectors, int32 dim, int32 pq_m, int32 pq_ks, int32 pq_subdim, int32 pq_code_bytes,
    const uint8* index_uuid, int index_uuidLen) {
  (void)h;
  // argument checks of retrieval_async_dsp_search.c:713-751
  if (!fd_pq_codes || !pq_chunk_vector_counts || !pq_codebook || !index_uuid || fd_pq_codesLen <= 0 ||
      fd_pq_codesLen > 64 || pq_chunk_vector_countsLen != fd_pq_codesLen || pq_chunk_vectors <= 0 ||
      num_vectors <= 0 || dim <= 0 || pq_m <= 0 || (pq_ks != 16 && pq_ks != 256) || pq_subdim <= 0 ||
      pq_m > INT32_MAX / pq_subdim || pq_m * pq_subdim != dim ||
      pq_code_bytes != (pq_ks == 16 ? pq_m / 2 + pq_m % 2 : pq_m) || index_uuidLen != 16)
    return AEE_EBADPARM;
  const size_t book = static_cast<size_t>(pq_m) * pq_ks * pq_subdim;
  if (book > static_cast<size_t>(INT32_MAX) || pq_codebookLen != static_cast<int>(book)) return AEE_EBADPARM;
  uint64_t total = 0;
  for (int i = 0; i < fd_pq_codesLen; ++i) {
    const int count = pq_chunk_vector_counts[i];
    if (fd_pq_codes[i] < 0 || count <= 0 || count > pq_chunk_vectors ||
        total > static_cast<uint64_t>(num_vectors) - static_cast<uint64_t>(count))
      return AEE_EBADPARM;
    if (i + 1 < fd_pq_codesLen && count != pq_chunk_vectors) return AEE_EBADPARM;
    total += count;
  }
  if (total != static_cast<uint64_t>(num_vectors)) return AEE_EBADPARM;
  for (size_t i = 0; i < book; ++i)
    if (!(pq_codebook[i] == pq_codebook[i]) || pq_codebook[i] > 3.402823466e+38F || pq_codebook[i] < -3.402823466e+38F)
      return AEE_EBADPARM;
  std::vector<uint8_t> codes(static_cast<size_t>(num_vectors) * pq_code_bytes);
  size_t done = 0;
  for (int i = 0; i < fd_pq_codesLen; ++i) {
    void* ptr = nullptr;
    size_t bytes = 0;
    const size_t want = static_cast<size_t>(pq_chunk_vector_counts[i]) * pq_code_bytes;
    if (rover_rpcmem_lookup(fd_pq_codes[i], &ptr, &bytes) != 0 || bytes < want) return AEE_EFAILED;
    std::memcpy(codes.data() + done, ptr, want);
    done += want;
  }
  RoverPqIndexDesc d{};
  d.num_vectors = num_vectors;
  d.graph_entry = -1;
  d.dim = dim;
  d.codes = codes.data();
  d.codebook = pq_codebook;
  d.m = pq_m;
  d.ks = pq_ks;
  d.subdim = pq_subdim;
  d.code_bytes = pq_code_bytes;
  const AEEResult r = calculator_rover_pq_load(h, &d);
  if (r == AEE_SUCCESS) {
    State& s = st();
    std::lock_guard<std::mutex> lock(s.mu);
    std::memcpy(s.pq_uuid, index_uuid, 16);
  }
  return r;
}

extern "C" AEEResult calculator_retrieval_pure_pq_unload_dma(remote_handle64 h) {
  return calculator_rover_pq_unload(h);
}

// The lane-protocol sessions (calculator_retrieval_pure_pq_sqmd_run,
// calculator_retrieval_expand_sqmd(_run)) are served by sessions.cu through
// the bridge below.

namespace rover {

bool session_acquire(SessionKind kind, SessionIndex* out) {
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (!s.init) {
    set_error("no index is loaded");
    return false;
  }
  if (s.session_live[kind] && kind != kSessionDb) {
    set_error("a session of this kind is already running");
    return false;
  }
  if (kind == kSessionPurePq) {
    if (!s.pq.loaded) {
      set_error("no pure-PQ index is loaded (calculator_retrieval_pure_pq_load_dma)");
      return false;
    }
    out->pq = s.pq.view;
    std::memcpy(out->pq_uuid, s.pq_uuid, 16);
  } else {
    if (!s.legacy.loaded) {
      set_error("no L1 index is loaded (calculator_retrieval_load / _load_dma)");
      return false;
    }
    out->sq = s.legacy.view;
    out->sq_graph_entry = s.legacy.graph_entry;
  }
  out->device = s.device;
  ++s.session_live[kind];
  return true;
}

void session_release(SessionKind kind) {
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  if (s.session_live[kind] > 0) --s.session_live[kind];
}

void session_count_launches(unsigned n) { g_launches += n; }

void session_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

}  // namespace rover

extern "C" AEEResult calculator_retrieval_async_submit(remote_handle64 h, const float* query, int queryLen,
                                                       const int* candidate_ids, int candidate_idsLen,
                                                       const uint8* compressed_batch, int compressed_batchLen,
                                                       int32 dim, int32 num_candidates, float scale, float zero_point,
                                                       int32* task_id) {
  (void)h; (void)query; (void)queryLen; (void)candidate_ids; (void)candidate_idsLen; (void)compressed_batch;
  (void)compressed_batchLen; (void)dim; (void)num_candidates; (void)scale; (void)zero_point;
  if (task_id) *task_id = -1;
  return AEE_EUNSUPPORTED;
}

extern "C" AEEResult calculator_retrieval_async_poll(remote_handle64 h, int32 task_id, int32* status, int* result_ids,
                                                     int result_idsLen, float* distances, int distancesLen,
                                                     int32* num_results) {
  (void)h; (void)task_id; (void)result_ids; (void)result_idsLen; (void)distances; (void)distancesLen;
  if (status) *status = 4;  // RETRIEVAL_ASYNC_DEMO_STATUS_NOT_FOUND
  if (num_results) *num_results = 0;
  return AEE_EUNSUPPORTED;
}

extern "C" AEEResult calculator_retrieval_async_reset(remote_handle64 h) {
  (void)h;
  return AEE_SUCCESS;
}

extern "C" AEEResult calculator_retrieval_rnn_l2_load_dma(remote_handle64 h, int32 fd_base, int32 num_vectors,
                                                          int32 dim) {
  (void)h; (void)fd_base; (void)num_vectors; (void)dim;
  return AEE_EUNSUPPORTED;
}

extern "C" AEEResult calculator_retrieval_rnn_l2_batch(remote_handle64 h, const int* ids_a, int ids_aLen,
                                                       const int* ids_b, int ids_bLen, int32 pair_count,
                                                       float* distances, int distancesLen) {
  (void)h; (void)ids_a; (void)ids_aLen; (void)ids_b; (void)ids_bLen; (void)pair_count; (void)distances;
  (void)distancesLen;
  return AEE_EUNSUPPORTED;
}

extern "C" AEEResult calculator_retrieval_rnn_l2_unload_dma(remote_handle64 h) {
  (void)h;
  return AEE_SUCCESS;
}

// ===========================================================================
// Allocation-free batched PQ search.
//
// For callers that may not allocate device memory at search time: a serving
// process whose memory pool already owns the whole GPU (a cudaMalloc there
// fails or fragments the pool), or a latency-critical loop that must not
// take cudaMalloc/cudaFree's implicit device synchronization.  The search
// kernel's scratch (the per-warp visited tables, the work counter and an
// error flag) lives in the fixed array below instead of library
// allocations.  The array is a static device variable: every GPU that loads
// this library holds its kNoAllocScratchBytes until the process exits.

namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;  // 64 MiB per device
constexpr size_t kNoAllocHeaderBytes = 256;           // work counter + error flag
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};   // device address of the array, per device
uint32_t g_noalloc_gen[kNoAllocMaxDevices] = {};         // next visited-table generation, per device
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// ORs every query status into one flag word.
__global__ void noalloc_status_any(const int32_t* status, int nq, unsigned int* flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    const int32_t s = status[i];
    if (s != kStatusOk) atomicOr(flag, 1u << (s & 31));
  }
}

}  // namespace

extern "C" AEEResult calculator_rover_pq_search_noalloc(remote_handle64 h, const RoverSearchParams* p,
                                                        const float* queries, int32_t nq,
                                                        const int32_t* pool_sizes, int32_t max_pool,
                                                        const int32_t* top_ks, const RoverSearchOutputs* out,
                                                        void* stream) {
  (void)h;
  if (!valid_params(p) || nq < 0 || !out || !queries || !pool_sizes || !out->status ||
      (out->ids && (!out->dists || !out->counts || out->out_stride <= 0)) ||
      (out->pool_ids && (!out->pool_dists || !out->pool_counts || p->pool_stride <= 0))) {
    set_error("invalid arguments: params, queries, pool_sizes and out->status are required, "
              "and each requested output needs its arrays and a positive stride");
    return AEE_EBADPARM;
  }
  // this entry runs the exact search over packed residual rows only
  if (p->mode != ROVER_MODE_EXACT || p->layout == ROVER_LAYOUT_DECODED || p->third_residual) {
    set_error("the no-alloc search runs mode ROVER_MODE_EXACT with the packed (or auto) layout and the "
              "mode-1 final refine only");
    return AEE_EBADPARM;
  }
  if (nq == 0) return AEE_SUCCESS;
  State& s = st();
  std::lock_guard<std::mutex> lock(s.mu);
  std::lock_guard<std::mutex> nlock(g_noalloc_mu);
  const PqDevice& pq = s.pq;
  if (!pq.loaded || !pq.has_graph) { set_error("no PQ index with a graph is loaded"); return AEE_EFAILED; }
  if (ensure_init(s) != AEE_SUCCESS) return AEE_EFAILED;   // refuses a device other than the index's
  if (max_pool <= 0 || max_pool > 4096) { set_error("max_pool must be in 1..4096"); return AEE_EBADPARM; }
  if (p->correction && pq.view.residual_bits == 0) { set_error("correction needs residuals"); return AEE_EBADPARM; }
  if (p->refine_budget > 0 && pq.view.residual_bits == 0) { set_error("refine needs residuals"); return AEE_EBADPARM; }
  if (p->third_residual && (!pq.view.e4.qparams || p->refine_budget <= 0)) {
    set_error("third_residual needs a loaded ERROR4 artifact and a refine budget");
    return AEE_EBADPARM;
  }
  const int expand = std::min(p->expand_count, pq.view.degree);
  if (expand > kMaxBatch) { set_error("expand_count above %d", kMaxBatch); return AEE_EBADPARM; }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) { set_error("device %d out of range", dev); return AEE_EFAILED; }
  cudaStream_t strm = static_cast<cudaStream_t>(stream);

  // Set-up, once per device, with that device current: the array's name is
  // a host-side stand-in in this code, so its device address must come from
  // cudaGetSymbolAddress before any kernel may be given it.
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      set_error("cudaGetSymbolAddress(no-alloc scratch) failed: %s", cudaGetErrorString(e));
      return AEE_EFAILED;
    }
    CK(cudaDeviceGetAttribute(&g_noalloc_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    CK(cudaMemsetAsync(ptr, 0, kNoAllocScratchBytes, strm));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(ptr);
    g_noalloc_gen[dev] = 1;
  }
  unsigned char* base = g_noalloc_ptr[dev];

  PqSearchArgs a{};
  a.ix = pq.view;
  a.queries = queries;
  a.nq = nq;
  a.pool_sizes = pool_sizes;
  a.top_ks = top_ks;
  a.top_k = p->top_k;
  a.entry_points = p->entry_points;
  a.graph_entry = pq.graph_entry;
  a.seed = p->seed;
  a.expand_count = p->expand_count;
  a.correction = p->correction;
  a.refine_budget = p->refine_budget;
  a.max_pool = max_pool;
  a.pool_ids = out->pool_ids;
  a.pool_dists = out->pool_dists;
  a.pool_stride = p->pool_stride;
  a.pool_counts = out->pool_counts;
  a.out_ids = out->ids;
  a.out_dists = out->dists;
  a.out_stride = out->out_stride;
  a.out_counts = out->counts;
  a.stats = reinterpret_cast<unsigned long long*>(out->stats);
  a.status = out->status;
  pq_search_layout(&a, p->refine_budget);
  const size_t smem = static_cast<size_t>(a.smem_per_warp) * kSearchWarps;
  if (smem > 227 * 1024) { set_error("shared memory %zu too large (pool %d)", smem, max_pool); return AEE_EBADPARM; }
  const PqSearchFn kernel = pq_search_kernel_for(pq.view, p->correction != 0);
  if (allow_smem(reinterpret_cast<const void*>(kernel), smem) != AEE_SUCCESS) return AEE_EFAILED;

  // Visited-table geometry: the same per-slot capacity rule as the
  // allocating path; the number of warp slots is what fits in the array.
  const uint64_t est = static_cast<uint64_t>(std::min(p->entry_points, pq.view.n)) +
                       (2ull * max_pool + 64ull) * static_cast<uint64_t>(expand);
  const uint32_t entries = next_pow2(std::max<uint64_t>(4096, 2 * est));
  const size_t per_slot = static_cast<size_t>(entries) * 8u;
  const size_t fit_slots = (kNoAllocScratchBytes - kNoAllocHeaderBytes) / per_slot;
  if (fit_slots < static_cast<size_t>(kSearchWarps)) {
    set_error("request needs %zu bytes of visited table per warp; the no-alloc scratch holds %zu bytes "
              "(%d warps minimum): lower pool/entry_points/expand_count or use calculator_rover_pq_search_device",
              per_slot, kNoAllocScratchBytes - kNoAllocHeaderBytes, kSearchWarps);
    return AEE_EBADPARM;
  }
  const int max_blocks = resident_blocks(reinterpret_cast<const void*>(kernel), kSearchWarps * 32, smem,
                                         g_noalloc_sms[dev]);
  int blocks = std::min<int>(max_blocks, static_cast<int>(fit_slots / kSearchWarps));
  blocks = std::max(1, std::min(blocks, (nq + kSearchWarps - 1) / kSearchWarps));

  // Generations make stale entries of earlier calls read as empty; when the
  // 32-bit range would wrap, the tables are cleared and numbering restarts.
  if (static_cast<uint64_t>(g_noalloc_gen[dev]) + static_cast<uint64_t>(nq) >= 0xffffffffull) {
    CK(cudaMemsetAsync(base + kNoAllocHeaderBytes, 0, kNoAllocScratchBytes - kNoAllocHeaderBytes, strm));
    g_noalloc_gen[dev] = 1;
  }
  a.visited = reinterpret_cast<unsigned long long*>(base + kNoAllocHeaderBytes);
  a.visited_mask = entries - 1u;
  a.gen_base = g_noalloc_gen[dev];
  g_noalloc_gen[dev] += static_cast<uint32_t>(nq);
  a.next_query = reinterpret_cast<unsigned int*>(base);
  unsigned int* flag = reinterpret_cast<unsigned int*>(base + 4);
  // the counter and the flag keep the last call's values: start them at zero
  CK(cudaMemsetAsync(base, 0, 8, strm));
  CK(cudaMemsetAsync(out->status, 0, static_cast<size_t>(nq) * sizeof(int32_t), strm));
  kernel<<<blocks, kSearchWarps * 32, smem, strm>>>(a);
  CK(cudaGetLastError());
  noalloc_status_any<<<std::min(64, (nq + 255) / 256), 256, 0, strm>>>(out->status, nq, flag);
  CK(cudaGetLastError());
  g_launches += 2;
  unsigned int any = 0;
  CK(cudaMemcpyAsync(&any, flag, sizeof(any), cudaMemcpyDeviceToHost, strm));
  CK(cudaStreamSynchronize(strm));
  if (any) {
    if (any & (1u << kStatusTableFull))
      set_error("a query exceeded its visited table (%u entries per warp) in the no-alloc scratch; "
                "rerun it with calculator_rover_pq_search_device", entries);
    else
      set_error("some queries failed: status bits 0x%x (see out->status)", any);
    return AEE_EFAILED;
  }
  return AEE_SUCCESS;
}
