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
// Entry seeds are ranked by ADC from the query's LUT (kept in shared memory)
// and only a shortlist of twice the pool is gated and merged.  The final
// refine (FP64, top refine_budget) runs as in every mode.
//
// The same kernel with beam width 1, full correction and a trace buffer
// writes the gate's training rows: every scored candidate and every
// expansion source with its features and whether it entered the pool.

#include <cfloat>
#include <cuda_bf16.h>

#include "pq_common.cuh"

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

// ADC distance from the query's LUT in shared memory (sequential sum over
// subspaces as retrieval_pq_adc_scalar, pq_core.c:392).
__device__ __forceinline__ float lut_adc(const PqIndexView& ix, const float* lut, int32_t id) {
  const uint8_t* code = ix.codes + static_cast<size_t>(id) * ix.code_bytes;
  float adc = 0.0f;
  if (ix.ks == 256 && (ix.m & 3) == 0) {
    for (int m0 = 0; m0 < ix.m; m0 += 4) {
      const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(code) + (m0 >> 2));
#pragma unroll
      for (int t = 0; t < 4; ++t) adc = fadd(adc, lut[(m0 + t) * 256 + ((w >> (8 * t)) & 255u)]);
    }
  } else {
    for (int m = 0; m < ix.m; ++m) {
      const int cc = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
      adc = fadd(adc, lut[m * ix.ks + cc]);
    }
  }
  return adc;
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

__device__ __forceinline__ void trace_put(const PqBatchArgs& c, int lane, bool have, const GateTraceRow& row) {
  const unsigned m = __ballot_sync(kFullMask, have);
  if (!m) return;
  unsigned long long start = 0;
  if (lane == 0) start = atomicAdd(c.trace_count, static_cast<unsigned long long>(__popc(m)));
  start = __shfl_sync(kFullMask, start, 0);
  if (have) {
    const unsigned long long idx = start + __popc(m & ((1u << lane) - 1u));
    if (idx < static_cast<unsigned long long>(c.trace_cap)) c.trace[idx] = row;
  }
}

// Position test after a merge: whether key (expanded bit clear) is in list.
__device__ __forceinline__ bool in_list(const uint64_t* list, int size, uint64_t key) {
  const int p = count_less(list, size, key);
  return p < size && key_cmp(list[p]) == key_cmp(key);
}

__device__ __forceinline__ void sort_merge_any(uint64_t* list, int* size, int cap, uint64_t* stage, int nb,
                                               int* cursor, int lane) {
  if (nb <= 32) sort_and_merge<1>(list, size, cap, stage, nb, cursor, lane);
  else if (nb <= 64) sort_and_merge<2>(list, size, cap, stage, nb, cursor, lane);
  else sort_and_merge<4>(list, size, cap, stage, nb, cursor, lane);
}

}  // namespace

template <int D, int KIND>
__global__ void __launch_bounds__(kSearchWarps * 32, 4)
pq_batched_search_kernel(PqSearchArgs a, PqDecodedArgs b, PqBatchArgs c) {
  constexpr bool kGated = KIND == kBatchGated;
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint8_t* base = smem + static_cast<size_t>(warp) * a.smem_per_warp;
  float* q = reinterpret_cast<float*>(base);
  uint64_t* list = reinterpret_cast<uint64_t*>(base + a.smem_query_bytes);
  uint64_t* stage = list + a.max_pool;
  int32_t* batch = reinterpret_cast<int32_t*>(stage + kMaxBatch);
  uint32_t* vis = reinterpret_cast<uint32_t*>(base + b.smem_vis_offset);
  const uint32_t vmask = static_cast<uint32_t>(b.vis_cap - 1);
  const bool tracing = c.trace != nullptr;
  const bool use_lut = kGated || tracing;
  uint64_t* shortl = use_lut ? reinterpret_cast<uint64_t*>(base + c.smem_short_offset) : nullptr;
  float* lut = use_lut ? reinterpret_cast<float*>(base + c.smem_lut_offset) : nullptr;
  uint32_t* feat = kGated ? reinterpret_cast<uint32_t*>(base + c.smem_feat_offset) : nullptr;
  float* logits = kGated ? reinterpret_cast<float*>(base + c.smem_logit_offset) : nullptr;
  const bool gate_on = kGated && c.gate.enabled;
  const int slot = blockIdx.x * kSearchWarps + warp;
  VisitedTable vt;
  vt.slots = a.visited + static_cast<size_t>(slot) * (a.visited_mask + 1ull);
  vt.mask = a.visited_mask;
  const PqIndexView& ix = a.ix;
  const int dim = D ? D : ix.dim;
  const float adc_bound = FLT_MAX / static_cast<float>(2 * ix.m);
  const int W = c.beam_width;

  for (;;) {
    int qi = 0;
    if (lane == 0) qi = b.q_begin + static_cast<int>(atomicAdd(a.next_query, 1u));
    qi = __shfl_sync(kFullMask, qi, 0);
    if (qi >= b.q_end) break;

    const int cap = a.pool_sizes[qi];
    int32_t* status = a.status + qi;
    const int expand = min(a.expand_count, ix.degree);
    if (cap <= 0 || cap > a.max_pool || expand <= 0 || W * expand > kMaxBatch || a.entry_points <= 0) {
      if (lane == 0) *status = kStatusBadParam;
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
    // LUT (retrieval_pq_build_lut); kept in shared memory when ADC is needed
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
      if (use_lut) lut[e] = acc;
    }
    if (__any_sync(kFullMask, bad)) {
      if (lane == 0) *status = kStatusNumeric;
      continue;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(kFullMask, lmax, off));
    const bool check_adc = !(lmax <= adc_bound);
    __syncwarp();
    vt.gen = a.gen_base + static_cast<uint32_t>(qi);
    int size = 0, cursor = 0;
    unsigned long long scored = static_cast<unsigned long long>(b.n_seeds), corrected = 0, expanded = 0;
    unsigned long long dedup = lane == 0 ? static_cast<unsigned long long>(b.seed_dups) : 0ull;
    int32_t st = kStatusOk;
    int scap = 0, ssize = 0;

    // ---- ADC shortlist of the seeds (gated search, traces)
    if (use_lut) {
      scap = min(c.short_cap, 2 * cap);
      int dummy = 0;
      for (int e0 = 0; e0 < b.n_seeds && st == kStatusOk; e0 += kMaxBatch) {
        const uint64_t thr = ssize == scap ? key_cmp(shortl[scap - 1]) : kEmptyKey;
        int cnt = 0;
        bool nonfinite = false;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int e = e0 + r * kWarp + lane;
          uint64_t k = kEmptyKey;
          if (e < b.n_seeds) {
            const int32_t id = __ldg(b.seed_ids + e);
            const float adc = lut_adc(ix, lut, id);
            if (!isfinite(adc)) nonfinite = true;
            else k = make_key(adc, id);
          }
          const bool keep = k < thr;
          const unsigned km = __ballot_sync(kFullMask, keep);
          if (keep) stage[cnt + __popc(km & ((1u << lane) - 1u))] = k;
          cnt += __popc(km);
        }
        if (__any_sync(kFullMask, nonfinite)) { st = kStatusNumeric; break; }
        __syncwarp();
        if (cnt) sort_merge_any(shortl, &ssize, scap, stage, cnt, &dummy, lane);
      }
    }

    if (!gate_on) {
      // ---- exact seed pool from the all-seeds distance pass
      corrected = static_cast<unsigned long long>(b.n_seeds);
      const float* drow = b.seed_dists + static_cast<size_t>(qi - b.q_begin) * b.n_seeds;
      for (int e0 = 0; e0 < b.n_seeds && st == kStatusOk; e0 += kMaxBatch) {
        const uint64_t thr = size == cap ? key_cmp(list[cap - 1]) : kEmptyKey;
        int cnt = 0;
        bool nonfinite = false;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int e = e0 + r * kWarp + lane;
          uint64_t k = kEmptyKey;
          if (e < b.n_seeds) {
            const float d = drow[e];
            if (!isfinite(d)) nonfinite = true;
            else k = make_key(d, __ldg(b.seed_ids + e));
          }
          const bool keep = k < thr;
          const unsigned km = __ballot_sync(kFullMask, keep);
          if (keep) stage[cnt + __popc(km & ((1u << lane) - 1u))] = k;
          cnt += __popc(km);
        }
        if (__any_sync(kFullMask, nonfinite)) { st = kStatusNumeric; break; }
        __syncwarp();
        if (cnt) sort_merge_any(list, &size, cap, stage, cnt, &cursor, lane);
      }
      if (st == kStatusOk && check_adc && !use_lut) {
        bool adc_bad = false;
        for (int e = lane; e < b.n_seeds; e += kWarp) {
          float adc, dist;
          if (!pq_score(ix, q, __ldg(b.seed_ids + e), false, &adc, &dist)) adc_bad = true;
        }
        if (__any_sync(kFullMask, adc_bad)) st = kStatusNumeric;
      }
      if (st == kStatusOk && tracing) {
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
      // ---- gated seeds: the shortlist, gated, merged into the pool
      const float worst = key_dist(shortl[min(ssize, cap) - 1]);
      for (int i0 = 0; i0 < ssize && st == kStatusOk; i0 += kMaxBatch) {
        const int nrow = min(kMaxBatch, ssize - i0);
        // decide: 0 keep ADC, 1 correct, 2 ask the MLP (row index in feat)
        int decision[kMaxBatch / kWarp];
        int nmlp = 0;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int i = i0 + r * kWarp + lane;
          int dcs = 0;
          if (i < i0 + nrow) {
            const float adc = key_dist(shortl[i]);
            const float ratio = adc / worst;
            dcs = ratio <= c.gate.band_lo ? 1 : (ratio >= c.gate.band_hi ? 0 : 2);
          }
          const unsigned mm = __ballot_sync(kFullMask, dcs == 2);
          if (dcs == 2) {
            const int row = nmlp + __popc(mm & ((1u << lane) - 1u));
            gate_row(c.gate, key_dist(shortl[i]), static_cast<float>(i) / cap, worst, 0.0f, qnorm, feat + row * 4);
            dcs = 2 + row;
          }
          nmlp += __popc(mm);
          decision[r] = dcs;
        }
        if (nmlp) gate_rows(c.gate, feat, nmlp, logits, lane);
        bool sbad = false;
        int ncorr = 0;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int i = i0 + r * kWarp + lane;
          if (i < i0 + nrow) {
            const uint64_t k = shortl[i];
            const int32_t id = key_id(k);
            int dcs = decision[r];
            if (dcs >= 2) dcs = logits[(dcs - 2) * 2] > c.gate.refine_logit ? 1 : 0;
            float d = key_dist(k);
            if (dcs == 1) {
              if (!row_dist<D>(b.decoded + static_cast<size_t>(id) * dim, q, dim, &d)) sbad = true;
              ++ncorr;
            }
            stage[i - i0] = make_key(d, id);
          }
        }
        if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) ncorr += __shfl_xor_sync(kFullMask, ncorr, off);
        corrected += ncorr;
        __syncwarp();
        sort_merge_any(list, &size, cap, stage, nrow, &cursor, lane);
      }
    }

    // ---- expansion steps
    bool global_mode = false;
    int claimed = 0;
    const uint32_t load_limit = (a.visited_mask + 1u) >> 1;
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
      if (gate_on) {
        // stop head on the selected sources
        if (lane < nsel) {
          int p = 0;
#pragma unroll
          for (int k = 0; k < kMaxBeamWidth; ++k)
            if (k == lane) p = sel[k];
          gate_row(c.gate, key_dist(list[p]), static_cast<float>(p) / cap, worst_now,
                   static_cast<float>(expanded) / cap, qnorm, feat + lane * 4);
        }
        gate_rows(c.gate, feat, nsel, logits, lane);
        float s = lane < nsel ? logits[lane * 2 + 1] : 0.0f;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(kFullMask, s, off);
        if (s / nsel > c.gate.stop_logit) break;
      }
      if (tracing) {
        int p = 0;
#pragma unroll
        for (int k = 0; k < kMaxBeamWidth; ++k)
          if (k == lane) p = sel[k];
        GateTraceRow row{};
        const bool have = lane < nsel;
        if (have) {
          const uint64_t k = list[p];
          row.query = qi; row.hop = static_cast<int32_t>(expanded) + lane; row.id = key_id(k); row.flags = 2;
          row.quantized = key_dist(k); row.rank = static_cast<float>(p) / cap; row.worst = worst_now;
          row.qnorm = qnorm; row.dist = key_dist(k);
        }
        trace_put(c, lane, have, row);
      }
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < nsel; ++k) list[sel[k]] |= kExpandedBit;
      cursor = sel[nsel - 1] + 1;
      // rows in pool order: valid prefix, then first visits
      int nb = 0;
      bool full = false, row_bad = false;
      for (int k = 0; k < nsel && !row_bad; ++k) {
        const int32_t src = key_id(list[sel[k]]);
        const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
        int first_pad = expand;
        int32_t nid_r[kMaxBatch / kWarp];
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int j = r * kWarp + lane;
          nid_r[r] = -1;
          if (r * kWarp < expand) {
            const int32_t nid = j < expand ? __ldg(row + j) : -1;
            nid_r[r] = nid;
            const unsigned pad = __ballot_sync(kFullMask, j < expand && nid == -1);
            if (pad && first_pad == expand) first_pad = r * kWarp + __ffs(pad) - 1;
          }
        }
        bool rb = false;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int j = r * kWarp + lane;
          if (j < expand) {
            const int32_t nid = nid_r[r];
            if (j < first_pad) rb |= (nid < 0 || nid >= ix.n);
            else rb |= (nid != -1);
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
        int fresh_here = 0;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          if (r * kWarp < first_pad) {
            const int j = r * kWarp + lane;
            int fresh = 0;
            const int32_t nid = nid_r[r];
            if (j < first_pad) {
              const uint32_t u = static_cast<uint32_t>(nid);
              if (__ldg(b.seed_bits + (u >> 5)) & (1u << (u & 31))) {
                ++dedup;
              } else {
                const int rr = global_mode ? visited_insert(vt, u) : smem_claim(vis, vmask, u);
                full |= rr < 0;
                fresh = rr == 1;
                if (rr == 0) ++dedup;
              }
            }
            const unsigned fm = __ballot_sync(kFullMask, fresh);
            if (fresh) batch[nb + __popc(fm & ((1u << lane) - 1u))] = nid;
            nb += __popc(fm);
            fresh_here += __popc(fm);
          }
        }
        claimed += fresh_here;
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
      // prefetch the candidates' decoded rows
      for (int e = lane; e < nb; e += kWarp) {
        const float* xr = b.decoded + static_cast<size_t>(batch[e]) * dim;
        for (int off = 0; off < dim; off += 32) asm volatile("prefetch.global.L1 [%0];" ::"l"(xr + off));
      }
      bool sbad = false;
      int ncorr = 0;
      if (!gate_on) {
        float adc_r[kMaxBatch / kWarp];
        for (int e = lane, r = 0; e < nb; e += kWarp, ++r) {
          const int32_t id = batch[e];
          float dist;
          if (!row_dist<D>(b.decoded + static_cast<size_t>(id) * dim, q, dim, &dist)) sbad = true;
          if (use_lut) {
            const float adc = lut_adc(ix, lut, id);
            if (!isfinite(adc)) sbad = true;
            adc_r[r] = adc;
          } else if (check_adc) {
            float adc, unused;
            if (!pq_score(ix, q, id, false, &adc, &unused)) sbad = true;
          }
          stage[e] = make_key(dist, id);
          ++ncorr;
        }
        if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
        if (tracing) {
          // features against the pool before this merge, kept in the
          // (otherwise unused) MLP scratch: ADC and rank per candidate
          float* tq = reinterpret_cast<float*>(base + c.smem_feat_offset);
          float* tr = tq + kMaxBatch;
          uint64_t* tk = reinterpret_cast<uint64_t*>(base + c.smem_logit_offset);
          for (int e = lane, r = 0; e < nb; e += kWarp, ++r) {
            const uint64_t k = stage[e];
            tq[e] = adc_r[r];
            tr[e] = static_cast<float>(count_less(list, size, make_key(adc_r[r], key_id(k)))) / cap;
            tk[e] = k;
          }
          __syncwarp();
          sort_merge_any(list, &size, cap, stage, nb, &cursor, lane);
          for (int e0 = 0; e0 < nb; e0 += kWarp) {
            const int e = e0 + lane;
            const bool have = e < nb;
            GateTraceRow row{};
            if (have) {
              const uint64_t k = tk[e];
              row.query = qi; row.hop = static_cast<int32_t>(expanded) - nsel; row.id = key_id(k);
              row.flags = in_list(list, size, k) ? 1 : 0;
              row.quantized = tq[e]; row.rank = tr[e]; row.worst = worst_now; row.qnorm = qnorm;
              row.dist = key_dist(k);
            }
            trace_put(c, lane, have, row);
          }
        } else {
          __syncwarp();
          sort_merge_any(list, &size, cap, stage, nb, &cursor, lane);
        }
      } else {
        // gated candidates: ADC, the band rule, the MLP inside the band
        const bool full_pool = size == cap;
        int decision[kMaxBatch / kWarp];
        float adc_r[kMaxBatch / kWarp];
        int nmlp = 0;
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int e = lane + r * kWarp;
          int dcs = 0;
          float adc = 0.0f;
          if (e < nb) {
            const int32_t id = batch[e];
            adc = lut_adc(ix, lut, id);
            if (!isfinite(adc)) sbad = true;
            const float ratio = full_pool ? adc / worst_now : 0.0f;
            dcs = ratio <= c.gate.band_lo ? 1 : (ratio >= c.gate.band_hi ? 0 : 2);
          }
          adc_r[r] = adc;
          const unsigned mm = __ballot_sync(kFullMask, dcs == 2);
          if (dcs == 2) {
            const int row = nmlp + __popc(mm & ((1u << lane) - 1u));
            const float rank = static_cast<float>(count_less(list, size, make_key(adc, batch[e]))) / cap;
            gate_row(c.gate, adc, rank, worst_now, static_cast<float>(expanded - nsel) / cap, qnorm, feat + row * 4);
            dcs = 2 + row;
          }
          nmlp += __popc(mm);
          decision[r] = dcs;
        }
        if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
        if (nmlp) gate_rows(c.gate, feat, nmlp, logits, lane);
#pragma unroll
        for (int r = 0; r < kMaxBatch / kWarp; ++r) {
          const int e = lane + r * kWarp;
          if (e < nb) {
            const int32_t id = batch[e];
            int dcs = decision[r];
            if (dcs >= 2) dcs = logits[(dcs - 2) * 2] > c.gate.refine_logit ? 1 : 0;
            float d = adc_r[r];
            if (dcs == 1) {
              if (!row_dist<D>(b.decoded + static_cast<size_t>(id) * dim, q, dim, &d)) sbad = true;
              ++ncorr;
            }
            stage[e] = make_key(d, id);
          }
        }
        if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
        __syncwarp();
        sort_merge_any(list, &size, cap, stage, nb, &cursor, lane);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) ncorr += __shfl_xor_sync(kFullMask, ncorr, off);
      corrected += ncorr;
    }

#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dedup += __shfl_xor_sync(kFullMask, dedup, off);
    if (st != kStatusOk) {
      if (lane == 0) *status = st;
      continue;
    }
    __syncwarp();
    pq_finish_query(a, q, list, size, qi, lane, base, scored, corrected, expanded, dedup);
    __syncwarp();
  }
}

PqBatchFn pq_batched_kernel_for(int dim, int kind) {
  if (dim % 4 != 0) return nullptr;
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
