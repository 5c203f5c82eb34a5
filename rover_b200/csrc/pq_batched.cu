// pq_batched.cu -- free-running batched PQ search and its learned gate.
//
// ROVER_MODE_BATCHED: the search of pq_decoded.cu (decoded rows, the
// all-seeds distance pass, the shared-memory visited table) except that each
// step expands the first `beam_width` unexpanded pool entries together: their
// rows are claimed in pool order, all fresh neighbours are corrected, sorted
// and merged in one pass.  With beam_width 1 this is the reference's own
// expansion order (retrieval_sqmd_pure_pq.c:867-934) and the results are the
// exact mode's; wider steps trade order for fewer serial steps.
//
// ROVER_MODE_GATED adds the learned gate, a 5 -> 64 -> 64 -> 2 MLP with BF16
// weights and FP32 accumulation, evaluated on warp-level tensor-core tiles
// (mma.sync m16n8k16, 16 rows per tile):
//   * refine head: per candidate, from its quantized (ADC) distance, its rank
//     in the pool, the pool's worst distance, the hop count and the query
//     norm, whether the candidate is corrected with its residual row; an
//     uncorrected candidate enters the pool with its ADC distance.  Only
//     candidates whose ADC / worst ratio lies inside (band_lo, band_hi) are
//     evaluated: below the band they are corrected, above it they keep ADC.
//   * stop head: per step, evaluated on the selected sources; when the mean
//     stop logit passes its threshold the query stops expanding.
// Entry seeds are ranked by their ADC distances (pq_seed_adc_kernel, one
// LUT per query in shared memory) and only a shortlist of twice the pool is
// gated and merged; expansion candidates are all corrected, since with
// decoded rows a correction costs what the in-place ADC it would be gated on
// costs.  The final refine (FP64, top refine_budget) runs as in every mode.
//
// The same kernel with beam width 1, full correction and a trace buffer
// writes the gate's training rows: every scored candidate and every
// expansion source with its features and whether it entered the pool.

#include <cfloat>
#include <cuda_bf16.h>

#include "pq_common.cuh"
#include "pq_seed_pool.cuh"

namespace rover {

namespace {

constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ int smem_claim(uint32_t* tab, uint32_t mask, uint32_t id) {
  uint32_t h = hash_id(id) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t prev = atomicCAS(tab + h, kEmpty, id);
    if (prev == kEmpty) return 1;
    if (prev == id) return 0;
    h = (h + 1) & mask;
  }
  return -1;
}

template <int D>
__device__ __forceinline__ bool row_dist(const float* __restrict__ xrow, const float* q, int dim, float* out) {
  const float4* x4 = reinterpret_cast<const float4*>(xrow);
  const float4* q4 = reinterpret_cast<const float4*>(q);
  const int n4 = D ? D / 4 : dim / 4;
  float acc = 0.0f;
#pragma unroll 8
  for (int t = 0; t < n4; ++t) {
    const float4 x = __ldg(x4 + t);
    const float4 qq = q4[t];
    float dl = fsub(qq.x, x.x); acc = fadd(acc, fmul(dl, dl));
    dl = fsub(qq.y, x.y); acc = fadd(acc, fmul(dl, dl));
    dl = fsub(qq.z, x.z); acc = fadd(acc, fmul(dl, dl));
    dl = fsub(qq.w, x.w); acc = fadd(acc, fmul(dl, dl));
  }
  *out = acc;
  return isfinite(acc);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Standardised gate inputs of one row, packed as four BF16x2 words.
__device__ __forceinline__ void gate_row(const GateParams& g, float quant, float rank, float worst, float hop,
                                         float qnorm, uint32_t* words) {
  const float x0 = (__logf(fmaxf(quant, 1e-30f)) - g.mu[0]) * g.inv_sigma[0];
  const float x1 = (rank - g.mu[1]) * g.inv_sigma[1];
  const float x2 = (__logf(fmaxf(worst, 1e-30f)) - g.mu[2]) * g.inv_sigma[2];
  const float x3 = (hop - g.mu[3]) * g.inv_sigma[3];
  const float x4 = (qnorm - g.mu[4]) * g.inv_sigma[4];
  words[0] = pack_bf16x2(x0, x1);
  words[1] = pack_bf16x2(x2, x3);
  words[2] = pack_bf16x2(x4, 0.0f);
  words[3] = 0u;
}

// One 16-row tile of the MLP: feat rows [row0, row0+16) (4 words each) ->
// logits[row][2].  The 13 KB of weights (transposed BF16 rows) are read
// through L1, where every warp of the SM shares them.
__device__ __noinline__ void gate_tile(const GateParams& gp, const uint32_t* feat, int row0, float* logits,
                                       int lane) {
  const uint32_t* __restrict__ w1 = reinterpret_cast<const uint32_t*>(gp.w1t);
  const uint32_t* __restrict__ w2 = reinterpret_cast<const uint32_t*>(gp.w2t);
  const uint32_t* __restrict__ w3 = reinterpret_cast<const uint32_t*>(gp.w3t);
  const float* __restrict__ b1 = gp.b1;
  const float* __restrict__ b2 = gp.b2;
  const float* __restrict__ b3 = gp.b3;
  constexpr int S1 = kGateW1Stride / 2, S2 = kGateW2Stride / 2;
  const int g = lane >> 2, t = lane & 3;
  const uint32_t a0 = feat[(row0 + g) * 4 + t];
  const uint32_t a1 = feat[(row0 + g + 8) * 4 + t];
  float h[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float c0 = __ldg(b1 + nt * 8 + 2 * t), c1 = __ldg(b1 + nt * 8 + 2 * t + 1);
    h[nt][0] = c0; h[nt][1] = c1; h[nt][2] = c0; h[nt][3] = c1;
    mma_bf16_16816(h[nt], a0, a1, 0u, 0u, __ldg(w1 + (nt * 8 + g) * S1 + t), 0u);
  }
  uint32_t A[4][4];
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    A[kk][0] = pack_bf16x2(fmaxf(h[2 * kk][0], 0.f), fmaxf(h[2 * kk][1], 0.f));
    A[kk][1] = pack_bf16x2(fmaxf(h[2 * kk][2], 0.f), fmaxf(h[2 * kk][3], 0.f));
    A[kk][2] = pack_bf16x2(fmaxf(h[2 * kk + 1][0], 0.f), fmaxf(h[2 * kk + 1][1], 0.f));
    A[kk][3] = pack_bf16x2(fmaxf(h[2 * kk + 1][2], 0.f), fmaxf(h[2 * kk + 1][3], 0.f));
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float c0 = __ldg(b2 + nt * 8 + 2 * t), c1 = __ldg(b2 + nt * 8 + 2 * t + 1);
    h[nt][0] = c0; h[nt][1] = c1; h[nt][2] = c0; h[nt][3] = c1;
    const uint32_t* wr = w2 + (nt * 8 + g) * S2;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma_bf16_16816(h[nt], A[kk][0], A[kk][1], A[kk][2], A[kk][3], __ldg(wr + kk * 8 + t),
                     __ldg(wr + kk * 8 + 4 + t));
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    A[kk][0] = pack_bf16x2(fmaxf(h[2 * kk][0], 0.f), fmaxf(h[2 * kk][1], 0.f));
    A[kk][1] = pack_bf16x2(fmaxf(h[2 * kk][2], 0.f), fmaxf(h[2 * kk][3], 0.f));
    A[kk][2] = pack_bf16x2(fmaxf(h[2 * kk + 1][0], 0.f), fmaxf(h[2 * kk + 1][1], 0.f));
    A[kk][3] = pack_bf16x2(fmaxf(h[2 * kk + 1][2], 0.f), fmaxf(h[2 * kk + 1][3], 0.f));
  }
  float o[4];
  o[0] = __ldg(b3 + 2 * t); o[1] = __ldg(b3 + 2 * t + 1); o[2] = o[0]; o[3] = o[1];
  const uint32_t* wr = w3 + g * S2;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk)
    mma_bf16_16816(o, A[kk][0], A[kk][1], A[kk][2], A[kk][3], __ldg(wr + kk * 8 + t), __ldg(wr + kk * 8 + 4 + t));
  if (t == 0) {
    logits[(row0 + g) * 2] = o[0];
    logits[(row0 + g) * 2 + 1] = o[1];
    logits[(row0 + g + 8) * 2] = o[2];
    logits[(row0 + g + 8) * 2 + 1] = o[3];
  }
}

__device__ __forceinline__ void gate_rows(const GateParams& gp, const uint32_t* feat, int nrows, float* logits,
                                          int lane) {
  __syncwarp();
  for (int r0 = 0; r0 < nrows; r0 += 16) gate_tile(gp, feat, r0, logits, lane);
  __syncwarp();
}

// Adds a search's MLP rows to the loaded gate's counter.
__device__ __forceinline__ void count_gate_rows(const GateParams& gp, int nrows, int lane) {
  if (lane == 0 && gp.rows_evaluated) atomicAdd(gp.rows_evaluated, static_cast<unsigned long long>(nrows));
}

// Appends the rows of the lanes that have one; returns this lane's row
// index, or ~0 when it wrote none (no row, or the buffer is full).
__device__ __forceinline__ unsigned long long trace_put(const PqBatchArgs& c, int lane, bool have,
                                                        const GateTraceRow& row) {
  const unsigned m = __ballot_sync(kFullMask, have);
  if (!m) return ~0ull;
  unsigned long long start = 0;
  if (lane == 0) start = atomicAdd(c.trace_count, static_cast<unsigned long long>(__popc(m)));
  start = __shfl_sync(kFullMask, start, 0);
  if (!have) return ~0ull;
  const unsigned long long idx = start + __popc(m & ((1u << lane) - 1u));
  if (idx >= static_cast<unsigned long long>(c.trace_cap)) return ~0ull;
  c.trace[idx] = row;
  return idx;
}

// Position test after a merge: whether key (expanded bit clear) is in list.
__device__ __forceinline__ bool in_list(const uint64_t* list, int size, uint64_t key) {
  const int p = count_less(list, size, key);
  return p < size && key_cmp(list[p]) == key_cmp(key);
}


}  // namespace

template <int D, int KIND>
__global__ void __launch_bounds__(kMaxSearchWarps * 32, 16 / kMaxSearchWarps)
pq_batched_search_kernel(PqSearchArgs a, PqDecodedArgs b, PqBatchArgs c) {
  constexpr bool kGated = KIND == kBatchGated;
  constexpr bool tracing = KIND == kBatchTrace;   // trace rows (full correction, beam width 1)
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint32_t* seed_filter = reinterpret_cast<uint32_t*>(smem);
  uint8_t* base = smem + b.filter_bits / 8 + static_cast<size_t>(warp) * a.smem_per_warp;
  float* q = reinterpret_cast<float*>(base);
  uint64_t* list = reinterpret_cast<uint64_t*>(base + a.smem_query_bytes);
  uint64_t* stage = list + a.max_pool;
  int32_t* batch = reinterpret_cast<int32_t*>(base + c.smem_ids_offset);   // kMaxBatchIds fresh ids per step
  uint32_t* vis = reinterpret_cast<uint32_t*>(base + b.smem_vis_offset);
  const uint32_t vmask = static_cast<uint32_t>(b.vis_cap - 1);
  constexpr bool adc_rows = kGated || tracing;     // quantized seed distances from pq_seed_rank_kernel
  uint64_t* shortl = adc_rows ? reinterpret_cast<uint64_t*>(base + c.smem_short_offset) : nullptr;
  uint32_t* feat = kGated ? reinterpret_cast<uint32_t*>(base + c.smem_feat_offset) : nullptr;
  float* logits = kGated ? reinterpret_cast<float*>(base + c.smem_logit_offset) : nullptr;
  const int slot = blockIdx.x * (blockDim.x >> 5) + warp;   // warps per CTA: set at launch
  VisitedTable vt;
  vt.slots = a.visited + static_cast<size_t>(slot) * (a.visited_mask + 1ull);
  vt.mask = a.visited_mask;
  const PqIndexView& ix = a.ix;
  const int dim = D ? D : ix.dim;
  const float adc_bound = FLT_MAX / static_cast<float>(2 * ix.m);
  const int W = c.beam_width;

  if (b.filter_bits) seed_filter_build(seed_filter, b.filter_bits, b.seed_ids, b.n_seeds);
  for (;;) {
    int item = 0;
    if (lane == 0) item = b.q_begin + static_cast<int>(atomicAdd(a.next_query, 1u));
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= b.q_end) break;
    // with an order, items index it and the seed rows cover every query
    const int qi = a.order ? __ldg(a.order + item) : item;
    const size_t seed_row_index = static_cast<size_t>(a.order ? qi : qi - b.q_begin);
    const size_t seed_row = seed_row_index * b.n_seeds;

    const int cap = a.pool_sizes[qi];
    int32_t* status = a.status + qi;
    const int expand = min(a.expand_count, ix.degree);
    if (cap <= 0 || cap > a.max_pool || expand <= 0 || expand > 2 * kWarp || W * expand > kMaxBatchIds ||
        a.entry_points <= 0) {
      if (lane == 0) *status = kStatusBadParam;
      continue;
    }
    if (b.seed_err && *reinterpret_cast<const volatile int*>(b.seed_err)) {
      if (lane == 0) *status = kStatusSeedRank;
      continue;
    }
    float qsq = 0.0f;
    {
      const float4* src = reinterpret_cast<const float4*>(a.queries + static_cast<size_t>(qi) * dim);
      for (int t = lane; t < dim / 4; t += kWarp) {
        const float4 v = __ldg(src + t);
        reinterpret_cast<float4*>(q)[t] = v;
        qsq += v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) qsq += __shfl_xor_sync(kFullMask, qsq, off);
    const float qnorm = sqrtf(qsq);
    for (int i = lane; i < b.vis_cap; i += kWarp) vis[i] = kEmpty;
    __syncwarp();
    bool check_adc = false;
    if (!lut_provably_safe(ix, q, lane)) {
      // retrieval_pq_build_lut fails the query on a non-finite LUT entry
      bool bad = false;
      float lmax = 0.0f;
      for (int e = lane; e < ix.m * ix.ks; e += kWarp) {
        const int m = e / ix.ks;
        const float* cen = ix.codebook + static_cast<size_t>(e) * ix.subdim;
        float acc = 0.0f;
        for (int j = 0; j < ix.subdim; ++j) {
          const float diff = fsub(q[m * ix.subdim + j], __ldg(cen + j));
          acc = fadd(acc, fmul(diff, diff));
        }
        if (!isfinite(acc)) bad = true;
        else lmax = fmaxf(lmax, acc);
      }
      if (__any_sync(kFullMask, bad)) {
        if (lane == 0) *status = kStatusNumeric;
        continue;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(kFullMask, lmax, off));
      check_adc = !(lmax <= adc_bound);
    }
    vt.gen = (a.gen_dev ? *a.gen_dev : a.gen_base) + static_cast<uint32_t>(qi);
    int size = 0, cursor = 0;
    unsigned long long scored = static_cast<unsigned long long>(b.n_seeds), corrected = 0, expanded = 0;
    unsigned long long dedup = lane == 0 ? static_cast<unsigned long long>(b.seed_dups) : 0ull;
    int32_t st = kStatusOk;
    int ssize = 0;

    // ---- ADC shortlist of the seeds (gated search, traces)
    if (adc_rows) {
      const int scap = min(c.short_cap, 2 * cap);
      const float* arow = c.seed_rank + seed_row_index * (c.rank_stride ? c.rank_stride : b.n_seeds);
      const float next = b.seed_top ? b.seed_top_next[seed_row_index] : 0.0f;
      if (b.seed_top && next == next && scap <= b.top_m) {
        // the row's top ranks, selected by pq_seed_topm_kernel: (rank, seed index) -> (rank, id)
        const uint64_t* top = b.seed_top + seed_row_index * b.top_m;
        ssize = min(scap, b.n_seeds);
        for (int i = lane; i < ssize; i += kWarp) {
          const uint64_t k = top[i];
          shortl[i] = make_key(key_dist(k), __ldg(b.seed_ids + key_id(k)));
        }
        __syncwarp();
      } else {
        int dummy = 0;
        const SeedRowKeys rk{arow, b.seed_ids};
        if (!(scap <= kMaxBatch ? select_top_lanes(shortl, &ssize, scap, stage, b.n_seeds, rk, &dummy, lane)
                                : select_top(shortl, &ssize, scap, stage, b.n_seeds, rk, &dummy, lane)))
          st = kStatusNumeric;
      }
    }

    if (!kGated) {
      // ---- exact seed pool: verified from the TF32 seed ranks (every pool
      // within kMaxBatch, not tracing), else from the all-seeds distance pass
      corrected = static_cast<unsigned long long>(b.n_seeds);
      if (!tracing && b.seed_verify) {
        const float* arow = b.seed_dists + seed_row_index * b.seed_stride;
        if (st == kStatusOk) {
          if (cap > kVerifyMaxPool) st = kStatusBadParam;
          else if (!verified_seed_pool<D>(list, &size, cap, stage, batch, b, arow,
                                          b.seed_top ? b.seed_top + seed_row_index * b.top_m : nullptr,
                                          b.seed_top ? b.seed_top_next[seed_row_index] : 0.0f, q, dim, &cursor,
                                          lane))
            st = kStatusNumeric;
        }
      } else {
        const float* drow = b.seed_dists + seed_row;
        if (st == kStatusOk &&
            !(cap <= kMaxBatch
                  ? select_top_lanes(list, &size, cap, stage, b.n_seeds, SeedRowKeys{drow, b.seed_ids}, &cursor, lane)
                  : select_top(list, &size, cap, stage, b.n_seeds, SeedRowKeys{drow, b.seed_ids}, &cursor, lane)))
          st = kStatusNumeric;
      }
      if (st == kStatusOk && check_adc) {
        bool adc_bad = false;
        for (int e = lane; e < b.n_seeds; e += kWarp) {
          float adc, dist;
          if (!pq_score(ix, q, __ldg(b.seed_ids + e), false, &adc, &dist)) adc_bad = true;
        }
        if (__any_sync(kFullMask, adc_bad)) st = kStatusNumeric;
      }
      if constexpr (tracing) if (st == kStatusOk) {
        // seed rows: the ADC shortlist with ranks among the seeds; label =
        // the seed is in the exact seed pool
        const float worst = key_dist(shortl[min(ssize, cap) - 1]);
        for (int i0 = 0; i0 < ssize; i0 += kWarp) {
          const int i = i0 + lane;
          GateTraceRow row{};
          const bool have = i < ssize;
          if (have) {
            const uint64_t k = shortl[i];
            const int32_t id = key_id(k);
            float dist = 0.0f;
            row_dist<D>(b.decoded + static_cast<size_t>(id) * dim, q, dim, &dist);
            row.query = qi; row.hop = 0; row.id = id;
            row.flags = 4 | (in_list(list, size, make_key(dist, id)) ? 1 : 0);
            row.quantized = key_dist(k); row.rank = static_cast<float>(i) / cap; row.worst = worst;
            row.qnorm = qnorm; row.dist = dist;
          }
          trace_put(c, lane, have, row);
        }
      }
    } else if (st == kStatusOk) {
      // ---- gated seeds: the shortlist, 32 rows at a time (one per lane)
      const float worst = key_dist(shortl[min(ssize, cap) - 1]);
      for (int i0 = 0; i0 < ssize && st == kStatusOk; i0 += kGateRows) {
        const int i = i0 + lane;
        const bool have = i < ssize;
        const uint64_t k = have ? shortl[i] : 0ull;
        const float adc = key_dist(k);
        const float ratio = adc / worst;
        int dcs = have ? (ratio <= c.gate.band_lo ? 1 : (ratio >= c.gate.band_hi ? 0 : 2)) : 0;
        const unsigned mm = __ballot_sync(kFullMask, dcs == 2);
        int row = 0;
        if (dcs == 2) {
          row = __popc(mm & ((1u << lane) - 1u));
          gate_row(c.gate, adc, static_cast<float>(i) / cap, worst, 0.0f, qnorm, feat + row * 4);
        }
        if (mm) {
          gate_rows(c.gate, feat, __popc(mm), logits, lane);
          count_gate_rows(c.gate, __popc(mm), lane);
        }
        if (dcs == 2) dcs = logits[row * 2] > c.gate.refine_logit ? 1 : 0;
        float d = adc;
        bool sbad = false;
        if (dcs == 1 && !row_dist<D>(b.decoded + static_cast<size_t>(key_id(k)) * dim, q, dim, &d)) sbad = true;
        if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
        corrected += __popc(__ballot_sync(kFullMask, dcs == 1));
        if (have) stage[lane] = make_key(d, key_id(k));
        __syncwarp();
        const int nrow = min(kGateRows, ssize - i0);
        merge_scored(list, &size, cap, stage, nrow, &cursor, lane);
      }
      if (lane != 0) corrected = 0;   // counted warp-wide; reduced with the lanes below
    }

    // ---- expansion steps
    bool global_mode = false;
    int claimed = 0;
    const uint32_t load_limit = (a.visited_mask + 1u) >> 1;
    unsigned long long ncorr_lane = 0;
    while (st == kStatusOk) {
      // the first W unexpanded entries
      int sel[kMaxBeamWidth];
      int nsel = 0;
      for (int b0 = cursor & ~31; b0 < size && nsel < W; b0 += kWarp) {
        const int i = b0 + lane;
        const bool cand = i >= cursor && i < size && !(list[i] & kExpandedBit);
        unsigned m = __ballot_sync(kFullMask, cand);
#pragma unroll
        for (int k = 0; k < kMaxBeamWidth; ++k) {
          if (m && nsel < W && k == nsel) {
            sel[k] = b0 + __ffs(m) - 1;
            m &= m - 1;
            ++nsel;
          }
        }
      }
      if (nsel == 0) break;
      const float worst_now = key_dist(list[size - 1]);
      int my_pos = 0;
#pragma unroll
      for (int k = 0; k < kMaxBeamWidth; ++k)
        if (k == lane && k < nsel) my_pos = sel[k];
      if (kGated && c.gate.stop_logit < FLT_MAX) {
        // stop head on the selected sources
        if (lane < nsel)
          gate_row(c.gate, key_dist(list[my_pos]), static_cast<float>(my_pos) / cap, worst_now,
                   static_cast<float>(expanded) / cap, qnorm, feat + lane * 4);
        gate_rows(c.gate, feat, nsel, logits, lane);
        count_gate_rows(c.gate, nsel, lane);
        float sl = lane < nsel ? logits[lane * 2 + 1] : 0.0f;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sl += __shfl_xor_sync(kFullMask, sl, off);
        if (sl / nsel > c.gate.stop_logit) break;
      }
      if constexpr (tracing) {
        GateTraceRow row{};
        const bool have = lane < nsel;
        if (have) {
          const uint64_t k = list[my_pos];
          row.query = qi; row.hop = static_cast<int32_t>(expanded) + lane; row.id = key_id(k); row.flags = 2;
          row.quantized = key_dist(k); row.rank = static_cast<float>(my_pos) / cap; row.worst = worst_now;
          row.qnorm = qnorm; row.dist = key_dist(k);
        }
        trace_put(c, lane, have, row);
      }
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < nsel; ++k) list[sel[k]] |= kExpandedBit;
      cursor = sel[nsel - 1] + 1;
      prefetch_next_rows(ix, list, size, cursor, W, lane);
      // the W rows, loaded together, then checked and claimed in pool order
      int32_t nid[kMaxBeamWidth][2];
#pragma unroll
      for (int k = 0; k < kMaxBeamWidth; ++k) {
        const int32_t src = k < nsel ? key_id(list[sel[k]]) : 0;
        const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int j = r * kWarp + lane;
          nid[k][r] = (k < nsel && j < expand) ? __ldg(row + j) : -1;
        }
      }
      int nb = 0;
      bool full = false, row_bad = false;
#pragma unroll 1
      for (int k = 0; k < nsel && !row_bad; ++k) {
        int first_pad = expand;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int j = r * kWarp + lane;
          const unsigned pad = __ballot_sync(kFullMask, j < expand && nid[k][r] == -1);
          if (pad && first_pad == expand) first_pad = r * kWarp + __ffs(pad) - 1;
        }
        bool rb = false;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int j = r * kWarp + lane;
          if (j < expand) {
            const int32_t v = nid[k][r];
            if (j < first_pad) rb |= (v < 0 || v >= ix.n);
            else rb |= (v != -1);
          }
        }
        if (__any_sync(kFullMask, rb)) { row_bad = true; break; }
        if (!global_mode && claimed + first_pad > b.vis_cap / 2) {
          for (int i = lane; i < b.vis_cap; i += kWarp) {
            const uint32_t id = vis[i];
            if (id != kEmpty && visited_insert(vt, id) < 0) full = true;
          }
          global_mode = true;
          __syncwarp();
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          if (r * kWarp < first_pad) {
            const int j = r * kWarp + lane;
            int fresh = 0;
            const int32_t v = nid[k][r];
            if (j < first_pad) {
              const uint32_t u = static_cast<uint32_t>(v);
              if (seed_filter_maybe(seed_filter, b.filter_bits, u) && (__ldg(b.seed_bits + (u >> 5)) & (1u << (u & 31)))) {
                ++dedup;
              } else {
                const int rr = global_mode ? visited_insert(vt, u) : smem_claim(vis, vmask, u);
                full |= rr < 0;
                fresh = rr == 1;
                if (rr == 0) ++dedup;
              }
            }
            const unsigned fm = __ballot_sync(kFullMask, fresh);
            if (fresh) batch[nb + __popc(fm & ((1u << lane) - 1u))] = v;
            nb += __popc(fm);
            claimed += __popc(fm);
          }
        }
      }
      if (row_bad) { st = kStatusBadRow; break; }
      expanded += nsel;
      if (__any_sync(kFullMask, full) || (global_mode && static_cast<uint32_t>(claimed) > load_limit)) {
        st = kStatusTableFull;
        break;
      }
      __syncwarp();
      if (nb == 0) continue;
      scored += nb;
      for (int e = lane; e < nb; e += kWarp) {
        const float* xr = b.decoded + static_cast<size_t>(batch[e]) * dim;
        for (int off = 0; off < dim; off += 32) asm volatile("prefetch.global.L1 [%0];" ::"l"(xr + off));
      }
      // every candidate corrected, scored and merged 128 at a time
      for (int c0 = 0; c0 < nb && st == kStatusOk; c0 += kMaxBatch) {
        const int cnt = min(kMaxBatch, nb - c0);
        bool sbad = false;
        for (int e = lane; e < cnt; e += kWarp) {
          const int32_t id = batch[c0 + e];
          float dist;
          if (!row_dist<D>(b.decoded + static_cast<size_t>(id) * dim, q, dim, &dist)) sbad = true;
          if (check_adc) {
            float adc, unused;
            if (!pq_score(ix, q, id, false, &adc, &unused)) sbad = true;
          }
          stage[e] = make_key(dist, id);
          ++ncorr_lane;
        }
        if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
        __syncwarp();
        if constexpr (tracing) {
          // rows before the merge (features against the current pool), the
          // entered flag patched after it
          unsigned long long tidx[kMaxBatch / kWarp];
          uint64_t keys[kMaxBatch / kWarp];
#pragma unroll
          for (int r = 0; r < kMaxBatch / kWarp; ++r) {
            const int e = lane + r * kWarp;
            const bool have = e < cnt;
            GateTraceRow row{};
            keys[r] = have ? stage[e] : 0ull;
            if (have) {
              const int32_t id = key_id(keys[r]);
              float adc = 0.0f, unused;
              pq_score(ix, q, id, false, &adc, &unused);
              row.query = qi; row.hop = static_cast<int32_t>(expanded) - nsel; row.id = id;
              row.quantized = adc;
              row.rank = static_cast<float>(count_less(list, size, make_key(adc, id))) / cap;
              row.worst = worst_now; row.qnorm = qnorm; row.dist = key_dist(keys[r]);
            }
            tidx[r] = r * kWarp < cnt ? trace_put(c, lane, have, row) : ~0ull;
          }
          __syncwarp();
          merge_scored(list, &size, cap, stage, cnt, &cursor, lane);
#pragma unroll
          for (int r = 0; r < kMaxBatch / kWarp; ++r)
            if (tidx[r] != ~0ull && in_list(list, size, keys[r])) c.trace[tidx[r]].flags = 1;
        } else {
          merge_scored(list, &size, cap, stage, cnt, &cursor, lane);
        }
      }
    }

#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      dedup += __shfl_xor_sync(kFullMask, dedup, off);
      ncorr_lane += __shfl_xor_sync(kFullMask, ncorr_lane, off);
    }
    if (kGated) corrected = __shfl_sync(kFullMask, corrected, 0);
    corrected += ncorr_lane;
    if (st != kStatusOk) {
      if (lane == 0) *status = st;
      continue;
    }
    __syncwarp();
    pq_finish_query(a, q, list, size, qi, lane, base, scored, corrected, expanded, dedup, b.decoded);
    __syncwarp();
  }
}

// The loaded gate on explicit rows, through the same feature packing and
// tensor-core tiles as the search: one warp per 32 rows.
__global__ void __launch_bounds__(128) gate_eval_kernel(GateParams g, const float* __restrict__ rows, int64_t n,
                                                        float* __restrict__ logits) {
  __shared__ uint32_t feat[4][32 * 4];
  __shared__ float out[4][32 * 2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t base = (static_cast<int64_t>(blockIdx.x) * 4 + warp) * 32;
  if (base >= n) return;
  const int64_t r = base + lane;
  if (r < n) {
    const float* x = rows + r * 5;
    gate_row(g, x[0], x[1], x[2], x[3], x[4], feat[warp] + lane * 4);
  } else {
    for (int k = 0; k < 4; ++k) feat[warp][lane * 4 + k] = 0u;
  }
  gate_rows(g, feat[warp], 32, out[warp], lane);
  if (r < n) {
    logits[r * 2] = out[warp][lane * 2];
    logits[r * 2 + 1] = out[warp][lane * 2 + 1];
  }
}

void launch_gate_eval(const GateParams& g, const float* rows, int64_t n, float* logits, cudaStream_t s) {
  const int64_t blocks = (n + 127) / 128;
  if (blocks > 0) gate_eval_kernel<<<static_cast<unsigned>(blocks), 128, 0, s>>>(g, rows, n, logits);
}

PqBatchFn pq_batched_kernel_for(int dim, int kind) {
  if (dim % 4 != 0) return nullptr;
  if (kind == kBatchTrace) return pq_batched_search_kernel<0, kBatchTrace>;
  if (kind == kBatchGated) {
    switch (dim) {
      case 128: return pq_batched_search_kernel<128, kBatchGated>;
      case 96: return pq_batched_search_kernel<96, kBatchGated>;
      default: return pq_batched_search_kernel<0, kBatchGated>;
    }
  }
  switch (dim) {
    case 128: return pq_batched_search_kernel<128, kBatchFull>;
    case 96: return pq_batched_search_kernel<96, kBatchFull>;
    default: return pq_batched_search_kernel<0, kBatchFull>;
  }
}

}  // namespace rover
