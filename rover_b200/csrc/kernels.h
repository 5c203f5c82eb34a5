// kernels.h -- launch-side view of the search and distance kernels.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace rover {

constexpr int kSearchWarps = 4;   // query warps per CTA (default)
constexpr int kMaxSearchWarps = 8;  // decoded / batched kernels take 1..8 warps per CTA (blockDim.x / 32)
constexpr int kMaxBatch = 128;    // max neighbours scored per expansion
constexpr int kVerifyMaxPool = 512;   // widest pool the verified seed pool serves (top-M of max(2L, L + 64))

struct PqSearchArgs {
  PqIndexView ix;
  const float* queries;          // [nq][dim], device
  int32_t nq;
  const int32_t* pool_sizes;     // [nq] beam width L per query
  const int32_t* top_ks;         // [nq] or null (then top_k)
  int32_t top_k;
  int32_t entry_points, graph_entry;
  uint32_t seed;
  int32_t expand_count;
  int32_t correction;
  int32_t refine_budget;         // 0 = no final refine
  int32_t third_residual;        // final refine in mode ERROR4 (ix.e4 loaded)
  int32_t max_pool;              // list capacity per warp (>= every pool size)
  // outputs (device)
  int32_t* pool_ids; float* pool_dists; int32_t pool_stride; int32_t* pool_counts;
  int32_t* out_ids; float* out_dists; int32_t out_stride; int32_t* out_counts;
  unsigned long long* stats;     // [nq][4] {scored, corrected, expanded, dedup}
  int32_t* status;               // [nq]
  // scratch (device)
  unsigned long long* visited;   // per warp slot: visited_mask + 1 entries
  uint32_t visited_mask;
  uint32_t gen_base;             // generation of query 0 (queries use gen_base + qi)
  const uint32_t* gen_dev;       // when set, the generation base is read here (plans: replays advance it)
  const int32_t* order;          // when set, claimed work item j serves query order[j]
  unsigned int* next_query;      // work counter, zero at launch
  // shared-memory layout per warp
  int32_t smem_per_warp, smem_query_bytes, smem_refine_offset, refine_capacity;
};

using PqSearchFn = void (*)(PqSearchArgs);
// The pq_search kernel instantiated for this index shape (a __global__
// function; launch with fn<<<grid, kSearchWarps * 32, smem, stream>>>(args)).
PqSearchFn pq_search_kernel_for(const PqIndexView& ix, bool correction);

// Layout of the per-warp shared-memory slice of pq_search_kernel.
inline void pq_search_layout(PqSearchArgs* a, int refine_budget) {
  const int qbytes = ((a->ix.dim * 4) + 15) & ~15;
  a->smem_query_bytes = qbytes;
  int off = qbytes + a->max_pool * 8 + kMaxBatch * 8 + kMaxBatch * 4;
  off = (off + 15) & ~15;
  a->smem_refine_offset = off;
  int cap = 0;
  if (refine_budget > 0) {
    cap = 1;
    while (cap < refine_budget) cap <<= 1;
  }
  a->refine_capacity = cap;
  a->smem_per_warp = (off + cap * 12 + 15) & ~15;
}

// ---- PQ search over decoded rows (correction on) ---------------------------
//
// The decoded layout stores every vector's residual reconstruction
// x = (c + code*s) + z as FP32 (NaN rows where the qparams are invalid), so a
// corrected distance is the plain sequential sum of (q - x)^2.  The entry
// seeds are the same for every query; their distances come from
// pq_seed_dists_kernel, a tiled all-queries x all-seeds pass.

struct PqDecodedArgs {
  const float* decoded;        // [n][dim]
  const int32_t* seed_ids;     // [n_seeds] distinct entry ids, draw order
  int32_t n_seeds;
  int32_t seed_dups;           // draws skipped as already visited
  const uint32_t* seed_bits;   // [ceil(n/32)] bitmap of seed ids
  const float* seed_dists;     // [q_end - q_begin][n_seeds]
  int32_t q_begin, q_end;      // queries served by this launch
  int32_t vis_cap;             // shared-memory visited slots per warp (power of two)
  int32_t smem_vis_offset;     // byte offset of that table in the warp slice
  int32_t filter_bits;         // seed filter at the start of the CTA's shared memory (power of two, 0 = none);
                               // the warp slices follow it
  int32_t seed_verify;         // 1: seed_dists holds TF32 ranks of the seeds' decoded rows (launch_pq_seed_rank
                               // over launch_pq_seed_gather's rows), verified exactly in the kernel; only
                               // with every pool size <= kMaxBatch
  const float* seed_norms;     // [n_seeds] |x_s|^2 of those rows (seed_verify)
  float seed_norm_max;         // their maximum (+inf if one is not finite)
  int32_t seed_stride;         // floats between seed_dists rows (0 = n_seeds); a multiple of 4 with seed_verify
  // per query row of the rank matrix (seed_verify, gated, traces): its top_m smallest keys (rank, seed index),
  // ascending, and the (top_m + 1)-th smallest rank (+inf when n_seeds <= top_m, NaN when the row held a
  // non-finite rank); null = select from the rank row in the search kernel
  const uint64_t* seed_top;
  const float* seed_top_next;
  int32_t top_m;
  // set by the tensor-core seed ranking when one of its bounded waits ran
  // out (search plans, which have no host check between the ranking and the
  // search): every query of the launch then fails with kStatusSeedRank
  const int* seed_err;
};

using PqDecodedFn = void (*)(PqSearchArgs, PqDecodedArgs);
// The decoded-layout kernel for this dimension (dim % 4 == 0 required).
PqDecodedFn pq_decoded_kernel_for(int dim);

// Warp slice: query | list | stage | batch | refine scratch | visited table.
inline void pq_decoded_layout(PqSearchArgs* a, PqDecodedArgs* b, int refine_budget, int vis_cap) {
  pq_search_layout(a, refine_budget);
  const int off = (a->smem_per_warp + 15) & ~15;
  b->smem_vis_offset = off;
  b->vis_cap = vis_cap;
  a->smem_per_warp = (off + vis_cap * 4 + 15) & ~15;
}

// ---- learned gate: 5 -> 64 -> 64 -> 2 MLP, BF16 weights, FP32 accumulation ----
//
// Inputs (standardised with mu / inv_sigma): log quantized distance, beam
// rank / L, log worst-in-beam distance, hop count / L, query norm.
// Outputs: refine-needed logit, stop-expanding logit.
constexpr int kGateIn = 5;
constexpr int kGateHidden = 64;
constexpr int kGateOut = 2;
constexpr int kGateW1Stride = 24;   // BF16 elements per transposed W1 row (16 used)
constexpr int kGateW2Stride = 72;   // BF16 elements per transposed W2 / W3 row (64 used)
constexpr int kMaxBeamWidth = 4;
constexpr int kMaxBatchIds = 256;  // fresh ids one batched step can claim (beam width x expand)

struct GateParams {
  const uint16_t* w1t;   // [64][24] BF16, W1 transposed (out x in), inputs 0..4
  const uint16_t* w2t;   // [64][72] BF16
  const uint16_t* w3t;   // [8][72]  BF16, rows 0..1 used
  const float* b1;       // [64]
  const float* b2;       // [64]
  const float* b3;       // [8]
  float mu[kGateIn], inv_sigma[kGateIn];
  float band_lo, band_hi;        // quantized / worst ratio: <= lo correct, >= hi keep, else MLP
  float refine_logit, stop_logit;
  int32_t enabled;               // 0: every candidate corrected, no early stop
  unsigned long long* rows_evaluated;   // MLP rows run inside searches (null: not counted)
};

// One trace row per scored candidate or expansion source (training data for
// the gate).  Written by the batched kernel with beam width 1 and full
// correction, i.e. along the reference's own expansion order.
struct GateTraceRow {
  int32_t query, hop, id, flags;   // flags: bit0 entered the pool, bit1 expansion source, bit2 seed
  float quantized, rank, worst, qnorm;
  float dist;                      // corrected distance
  float pad[3];
};

struct PqBatchArgs {
  int32_t beam_width;
  GateParams gate;
  GateTraceRow* trace;            // null = no trace
  unsigned long long* trace_count;
  int64_t trace_cap;
  const float* seed_rank;         // [q_end - q_begin][rank_stride] quantized seed distances (gated, traces)
  int32_t rank_stride;            // floats between seed_rank rows (0 = n_seeds)
  int32_t short_cap;              // gated seeds: ADC shortlist capacity
  int32_t smem_ids_offset, smem_short_offset, smem_feat_offset, smem_logit_offset;
};

enum PqBatchKind : int { kBatchFull = 0, kBatchGated = 1, kBatchTrace = 2 };
using PqBatchFn = void (*)(PqSearchArgs, PqDecodedArgs, PqBatchArgs);
PqBatchFn pq_batched_kernel_for(int dim, int kind);

constexpr int kGateRows = 32;    // MLP rows per warp pass (one per lane)

// Batched warp slice: the decoded slice, the step's fresh ids, then (gated
// or traced) the seed shortlist, MLP features (BF16 [32][8]) and logits
// ([32][2]).
inline void pq_batched_layout(PqSearchArgs* a, PqDecodedArgs* b, PqBatchArgs* c, int refine_budget, int vis_cap,
                              bool gate_rows) {
  pq_decoded_layout(a, b, refine_budget, vis_cap);
  int off = a->smem_per_warp;
  c->smem_ids_offset = off;
  off += kMaxBatchIds * 4;
  if (gate_rows) {
    c->smem_short_offset = off;
    off += c->short_cap * 8;
    c->smem_feat_offset = off;
    off += kGateRows * 8 * 2;
    c->smem_logit_offset = off;
    off += kGateRows * 2 * 4;
  }
  a->smem_per_warp = (off + 15) & ~15;
}

void launch_pq_decode(const PqIndexView& ix, float* decoded, cudaStream_t s);
void launch_pq_seed_dists(const float* queries, int q_begin, int q_end, int dim, const float* decoded,
                          const int32_t* seed_ids, int n_seeds, float* out, cudaStream_t s);
// Seed PQ reconstructions [n_seeds][dim] and their squared norms.
// Per row of a queries x seeds rank matrix (row stride `stride`): the m
// smallest keys (rank, seed index) ascending into keys[row][m] and the
// (m + 1)-th smallest rank into next[row] (+inf if n_seeds <= m, NaN if the
// row holds a rank of 3e38 or more, or more than 2,048 ranks tie with the
// (m + 1)-th).  One CTA per row.
void launch_pq_seed_topm(const float* rank, int stride, int n_seeds, int rows, int m, uint64_t* keys, float* next,
                         cudaStream_t s);
inline int seed_top_m(int n_seeds, int max_pool) {
  const int m = std::max(2 * max_pool, max_pool + 64);
  return std::min(n_seeds, std::min(1024, (m + 31) / 32 * 32));
}

// rows[u] = decoded[seed_ids[u]], norms[u] = |rows[u]|^2 (FP32).
void launch_pq_seed_gather(const float* decoded, int dim, const int32_t* seed_ids, int n_seeds, float* rows,
                           float* norms, cudaStream_t s);
void launch_pq_seed_recon(const PqIndexView& ix, const int32_t* seed_ids, int n_seeds, float* rows, float* norms,
                          cudaStream_t s);
// Quantized seed distances for ranking (TF32 tensor cores):
// out[q - q_begin][u] = |q|^2 + |x~_u|^2 - 2 q . x~_u.  dim % 4 == 0.
// The same ranks on tcgen05 tensor cores (seed_rank_tc.cu) for dim in
// {32, 64, 96, 128}: the seed rows are a TF32-rounded copy named by a TMA
// descriptor.  *err is set if a bounded wait inside the kernel ran out.
struct alignas(64) TcSeedMap {
  unsigned char bytes[128];   // CUtensorMap
  int32_t valid;
};
bool seed_rank_tc_supported(int dim);
bool tc_seed_map_encode(TcSeedMap* m, const float* rows_tf32, int n_seeds, int dim);
void launch_tf32_round(const float* in, float* out, size_t n, cudaStream_t s);
void launch_row_norms(const float* rows, int n, int dim, float* norms, cudaStream_t s);
bool launch_pq_seed_rank_tc(const TcSeedMap& m, const float* queries, int q_begin, int q_end, int dim,
                            const float* norms, int n_seeds, float* out, int out_stride, int* err, int sms,
                            cudaStream_t s);
void launch_pq_seed_rank(const float* queries, int q_begin, int q_end, int dim, const float* rows, const float* norms,
                         int n_seeds, float* out, cudaStream_t s, int out_stride = 0);   // 0: rows of n_seeds

// ---- search plans (plan.cu) --------------------------------------------------
//
// A plan replays the same searches on new query vectors, possibly from a
// captured CUDA graph, so the per-launch bookkeeping lives on the device: the
// generation base of the launch's visited-table tags, a flag asking for the
// tables to be cleared when the next launch's tags would wrap, and one work
// counter per beam-width class.

constexpr int kMaxPlanClasses = 8;

struct PlanControl {
  uint32_t gen;                          // generation of query 0 in the next launch
  uint32_t clear;                        // 1: zero the visited tables before the next launch
  uint32_t counters[kMaxPlanClasses];    // work counters of the class launches
};

// Zeroes the class counters and status[0, nq), and the visited tables when
// ctl->clear is set.
void launch_plan_prepare(PlanControl* ctl, unsigned long long* visited, size_t visited_words, int32_t* status, int nq,
                         int classes, int sms, cudaStream_t s);
// Moves ctl->gen past this launch's nq generations; asks for a clear when
// the next launch's generations would pass 2^32 - 1.
void launch_plan_advance(PlanControl* ctl, int nq, cudaStream_t s);

// The gate's logits [n][2] of raw rows [n][5] (quantized distance, rank / L,
// worst distance, hop / L, query norm), as the batched search evaluates them.
void launch_gate_eval(const GateParams& g, const float* rows, int64_t n, float* logits, cudaStream_t s);

// ---- gate training (gate_train.cu) ------------------------------------------
void launch_gate_stats(const float* x, int64_t n, double* acc, cudaStream_t s);
cudaError_t launch_gate_fwd_bwd(const float* params, const float* mu, const float* sigma, const float* x,
                                const float* y, const float* m, const int64_t* idx, int64_t n, float pw0, float pw1,
                                float denom, float* grad, double* loss, cudaStream_t s);
void launch_gate_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2,
                      float eps, float wd, float bc1, float bc2, cudaStream_t s);

// ---- SQ search (heap-exact) ----------------------------------------------

enum SqSearchMode : int32_t { kSqModeDsp = 0, kSqModeSqmd = 1, kSqModeDb = 2 };

struct SqSearchArgs {
  SqIndexView ix;
  const float* queries; int32_t nq;
  const int32_t* pool_sizes;
  int32_t mode;                  // kSqModeDsp (a15), kSqModeSqmd (a12) or kSqModeDb (DB-pair)
  int32_t entry_points, graph_entry;
  uint32_t seed;
  int32_t expand_count;
  int32_t correction;            // SQMD only
  int32_t split;                 // SQMD with the SQ4 split distance (ix.split_bias)
  int32_t num_out;               // DSP mode: outputs per query
  int32_t max_pool;              // pool heap capacity per slot
  int32_t frontier_cap;          // frontier heap capacity per slot
  int32_t* out_ids; float* out_dists; int32_t out_stride; int32_t* out_counts;
  unsigned long long* stats;     // [nq][4]
  int32_t* status;
  unsigned long long* visited; uint32_t visited_mask; uint32_t gen_base;
  uint64_t* heaps;               // per slot: max_pool + frontier_cap entries
  unsigned int* next_query;
  // the request's entry ids, the same for every query (drawn on the host):
  // DSP / DB-pair: entry_points ids in draw order, repeats included;
  // SQMD: the distinct seeds of retrieval_sqmd_make_seed_ids
  const int32_t* entry_ids; int32_t entry_count;
  // heap entries kept in shared memory per warp (the rest at the same
  // indices of the slot's global heaps)
  int32_t pool_split, front_split;
};

using SqSearchFn = void (*)(SqSearchArgs);
// Dynamic shared memory of one warp of the SQ search kernel.
size_t sq_search_smem_per_warp(int dim, int pool_split, int front_split);
// The SQ search kernel (a __global__ function): with the split distance
// compiled in or out, so the plain searches keep their register budget.
SqSearchFn sq_search_kernel_for(bool split);

// ---- DB-pair search driven step by step by the host (calculator_retrieval_search_db)
//
// Two queries (slots), each one search of the reference's DB-pair loop
// (retrieval_async_dsp_search.c:1205-1581) kept on the device; the host
// drives it one step at a time through the shared expansion buffers, because
// each expansion waits for the caller's corrected distances.
constexpr int kDbSlots = 2;
constexpr int kDbItems = 32;     // DB_MAX_EXPAND
enum DbOp : int32_t { kDbNone = 0, kDbInit = 1, kDbStep = 2, kDbFinish = 3 };

struct DbIo {                    // host <-> device per launch (pinned twin on the host)
  int32_t op[kDbSlots];
  int32_t count[kDbSlots];       // in (kDbStep): corrections for the last step's ids; out: this step's ids
  float corr[kDbSlots][kDbItems];
  int32_t ids[kDbSlots][kDbItems];
  float coarse[kDbSlots][kDbItems];
  int32_t finished[kDbSlots];
  int32_t status[kDbSlots];
  int32_t out_count[kDbSlots];   // kDbFinish
};

struct DbSlot {                  // device-resident search state of one query
  int32_t psize, fsize, finished, last_count;
  int32_t last_ids[kDbItems];
  uint8_t qc[1024];
};

struct DbArgs {
  SqIndexView ix;
  const float* queries;          // [kDbSlots][dim]
  int32_t entry_points, expand_limit, pool_cap, num_out, graph_entry, frontier_cap;
  DbIo* io;
  DbSlot* slots;
  uint64_t* pools;               // [kDbSlots][pool_cap] (id, dist) pairs
  uint64_t* fronts;              // [kDbSlots][frontier_cap]
  uint32_t* visited;             // [kDbSlots][(n + 31) / 32]
  int32_t* out_ids;              // [kDbSlots][num_out]
  float* out_dists;
};
void launch_db_step(const DbArgs& a, cudaStream_t s);

// ---- batched distance kernels ---------------------------------------------

void launch_pq_lut(const PqIndexView& ix, const float* queries, int nq, float* luts,
                   int32_t* status, cudaStream_t s);
void launch_pq_adc(const PqIndexView& ix, const float* luts, int nq, const int32_t* ids,
                   const int64_t* offsets, float* out, int32_t* status, cudaStream_t s);
void launch_pq_residual(const PqIndexView& ix, const float* queries, int nq, const int32_t* ids,
                        const int64_t* offsets, float* out, int32_t* status, cudaStream_t s);
void launch_pq_rescore(int dim, int n, const float* decoded, const float* queries, int nq, const int32_t* ids,
                       const int64_t* offsets, float* out, int32_t* status, cudaStream_t s);
void launch_sq_coarse(const SqIndexView& ix, const float* queries, int nq, const int32_t* ids,
                      const int64_t* offsets, float* out, int32_t* status, cudaStream_t s);
void launch_sq_exact(const SqIndexView& ix, const float* queries, int nq, const int32_t* ids,
                     const int64_t* offsets, float* out, int32_t* status, cudaStream_t s);
// demo_rerank_candidates on the SQ index (capacity <= 4096 candidates).
void launch_rerank(const SqIndexView& ix, const float* queries, int nq, const int32_t* cand_ids, int cand_stride,
                   const int32_t* cand_counts, int top_k, int capacity, int32_t* out_ids, float* out_dists,
                   int32_t* out_counts, int32_t* status, cudaStream_t s);
// decoded: the PQ index's decoded rows (kind 1, dim % 4 == 0) or null.
// error4: mode ERROR4, the index view's e4 term added to every decode.
void launch_refine(int kind, const PqIndexView& pq, const SqIndexView& sq, const float* decoded, const float* queries,
                   int nq, const int32_t* cand_ids, int cand_stride, const int32_t* cand_counts,
                   int top_k, int capacity, int32_t* out_ids, float* out_dists,
                   int32_t* out_counts, int32_t* status, cudaStream_t s, bool error4 = false);
// The split distance's lane part (retrieval_compute_u8_u4_l1_distance) of
// ids[offsets[q]..offsets[q+1]) against the aligned u8 queries [nq][dim].
void launch_sq_aligned_coarse(const SqIndexView& ix, const uint8_t* queries_u8, int nq, const int32_t* ids,
                              const int64_t* offsets, float* out, int32_t* status, cudaStream_t s);

// ---- PQ codebook training and encoding (pq_train.cu)
//
// retrieval_pq_train (retrieval_pq_core.c:97-224) over x [n][dim] on the
// device, all m subspaces at once; book [m][ks][dim/m] receives the
// codebook.  The scratch (assignments, per-block histograms, member lists)
// is owned by the caller's PqTrainScratch.
struct PqTrainScratch {
  uint8_t* assign = nullptr;
  int* block_hist = nullptr;
  int* counts = nullptr;
  int* members = nullptr;
  ~PqTrainScratch();
  void release();
};
cudaError_t pq_train_device(const float* x, int n, int dim, int m, int ks, int iters, float* book,
                            PqTrainScratch* scratch, cudaStream_t s);
int pq_train_launches(int iters);
// retrieval_pq_encode_batch (:226-268): codes [n][code_bytes], 4-bit codes
// packed low nibble first when ks <= 16; *bad = 1 on a non-finite distance.
void launch_pq_encode(const float* x, long long n, int dim, int m, int ks, const float* book, uint8_t* codes,
                      int* bad, cudaStream_t s);

}  // namespace rover
