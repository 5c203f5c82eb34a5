// pq_common.cuh -- PQ scoring, pool merge and refine helpers shared by the
// PQ search kernels (packed-residual and decoded-row layouts).
//
// Sources followed: retrieval_pq_build_lut / retrieval_pq_adc_scalar
// (src/imp/retrieval_pq_core.c:362, :392), retrieval_pq_residual_query_evaluate
// (src/dsp_demo/retrieval_pq_residual.c:983) and refine_impl
// (src/dsp_demo/retrieval_final_refine.c:256-292).
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace rover {

// Residual row address inside the .pqresN block payload
// (pq_residual_query_block, retrieval_pq_residual.c:914-924).
__device__ __forceinline__ const uint8_t* pq_residual_row(const PqIndexView& ix, int32_t id) {
  const uint32_t u = static_cast<uint32_t>(id);
  const uint32_t block = u / static_cast<uint32_t>(ix.vpb);
  const uint32_t within = (u - block * static_cast<uint32_t>(ix.vpb)) * static_cast<uint32_t>(ix.rcb);
  return ix.residual + static_cast<size_t>(block) * 4096u + within;
}

// One candidate's ADC distance (retrieval_pq_build_lut entries recomputed in
// place, then the sequential sum of retrieval_pq_adc_scalar) and, when
// correction is on, the residual-corrected distance.  Returns false when the
// reference would reject the candidate (non-finite or invalid qparams).
__device__ __forceinline__ bool pq_score(const PqIndexView& ix, const float* __restrict__ q,
                                         int32_t id, bool correction, float* out_adc,
                                         float* out_dist) {
  const uint8_t* code = ix.codes + static_cast<size_t>(id) * ix.code_bytes;
  float adc = 0.0f;
  float acc = 0.0f;
  float scale = 0.0f, zero = 0.0f;
  const uint8_t* res = nullptr;
  if (correction) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    scale = qp.x;
    zero = qp.y;
    if (!isfinite(scale) || !isfinite(zero) || !(scale > 0.0f)) return false;
    res = pq_residual_row(ix, id);
  }
  int dim = 0;
  for (int m = 0; m < ix.m; ++m) {
    const int c = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
    const float* cen = ix.codebook + (static_cast<size_t>(m) * ix.ks + c) * ix.subdim;
    float lut = 0.0f;
    for (int j = 0; j < ix.subdim; ++j, ++dim) {
      const float cj = __ldg(cen + j);
      const float qd = q[dim];
      const float diff = fsub(qd, cj);
      lut = fadd(lut, fmul(diff, diff));
      if (correction) {
        const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, dim))
                                                 : static_cast<uint32_t>(__ldg(res + dim));
        const float x = fadd(fadd(cj, fmul(u8f(r), scale)), zero);
        const float dq = fsub(qd, x);
        acc = fadd(acc, fmul(dq, dq));
      }
    }
    adc = fadd(adc, lut);
  }
  if (!isfinite(adc)) return false;
  if (correction && !isfinite(acc)) return false;
  *out_adc = adc;
  *out_dist = correction ? acc : adc;
  return true;
}

// Shape-specialised scorer for Ks=256 codebooks: the candidate's whole code
// row and residual row are fetched up front with 16-byte (or 8/4-byte)
// vector loads and every loop is unrolled, so a candidate costs one round
// of independent memory requests instead of one per subspace or dimension.
// The floating-point operations and their order are those of pq_score.
template <int M, int SUB, int RBITS>
__device__ __forceinline__ bool pq_score_fixed(const PqIndexView& ix, const float* __restrict__ q, int32_t id,
                                               bool correction, float* out_adc, float* out_dist) {
  constexpr int DIM = M * SUB;
  constexpr int RCB = RBITS == 8 ? DIM : DIM / 2;
  constexpr int CW = (M + 3) / 4;      // code words
  constexpr int RW = RCB / 4;          // residual words
  uint32_t cw[CW];
  const uint8_t* crow = ix.codes + static_cast<size_t>(id) * M;
  if constexpr (M % 16 == 0) {
#pragma unroll
    for (int i = 0; i < M / 16; ++i) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(crow) + i);
      cw[4 * i] = v.x; cw[4 * i + 1] = v.y; cw[4 * i + 2] = v.z; cw[4 * i + 3] = v.w;
    }
  } else if constexpr (M % 8 == 0) {
#pragma unroll
    for (int i = 0; i < M / 8; ++i) {
      const uint2 v = __ldg(reinterpret_cast<const uint2*>(crow) + i);
      cw[2 * i] = v.x; cw[2 * i + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < CW; ++i) cw[i] = __ldg(reinterpret_cast<const uint32_t*>(crow) + i);
  }
  uint32_t rw[RW];
  float scale = 0.0f, zero = 0.0f;
  if (correction) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    scale = qp.x;
    zero = qp.y;
    const uint8_t* res = pq_residual_row(ix, id);
    if constexpr (RCB % 16 == 0) {
#pragma unroll
      for (int i = 0; i < RCB / 16; ++i) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(res) + i);
        rw[4 * i] = v.x; rw[4 * i + 1] = v.y; rw[4 * i + 2] = v.z; rw[4 * i + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int i = 0; i < RW; ++i) rw[i] = __ldg(reinterpret_cast<const uint32_t*>(res) + i);
    }
    if (!isfinite(scale) || !isfinite(zero) || !(scale > 0.0f)) return false;
  }
  float adc = 0.0f, acc = 0.0f;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const uint32_t c = (cw[m >> 2] >> (8 * (m & 3))) & 255u;
    const float* cen = ix.codebook + (static_cast<size_t>(m) * 256u + c) * SUB;
    float cv[SUB];
    if constexpr (SUB % 4 == 0) {
#pragma unroll
      for (int t = 0; t < SUB / 4; ++t) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(cen) + t);
        cv[4 * t] = v.x; cv[4 * t + 1] = v.y; cv[4 * t + 2] = v.z; cv[4 * t + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int t = 0; t < SUB; ++t) cv[t] = __ldg(cen + t);
    }
    float lut = 0.0f;
#pragma unroll
    for (int j = 0; j < SUB; ++j) {
      const int d = m * SUB + j;
      const float qd = q[d];
      const float diff = fsub(qd, cv[j]);
      lut = fadd(lut, fmul(diff, diff));
      if (correction) {
        uint32_t r;
        if constexpr (RBITS == 8) r = (rw[d >> 2] >> (8 * (d & 3))) & 255u;
        else r = (rw[d >> 3] >> (4 * (d & 7))) & 15u;
        const float x = fadd(fadd(cv[j], fmul(u8f(r), scale)), zero);
        const float dq = fsub(qd, x);
        acc = fadd(acc, fmul(dq, dq));
      }
    }
    adc = fadd(adc, lut);
  }
  if (!isfinite(adc)) return false;
  if (correction && !isfinite(acc)) return false;
  *out_adc = adc;
  *out_dist = correction ? acc : adc;
  return true;
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

// Residual-corrected distance (retrieval_pq_residual_query_evaluate) of
// one candidate whose code row and residual row are given as 32-bit words
// (wherever they were loaded from): the operations and order of pq_score.
// False when the reference rejects the candidate.
template <int M, int SUB, int RBITS>
__device__ __forceinline__ bool pq_residual_words(const PqIndexView& ix, const float* __restrict__ q,
                                                  const uint32_t* cw, const uint32_t* rw, float2 qp,
                                                  float* out_dist) {
  if (!isfinite(qp.x) || !isfinite(qp.y) || !(qp.x > 0.0f)) return false;
  float acc = 0.0f;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const uint32_t c = (cw[m >> 2] >> (8 * (m & 3))) & 255u;
    const float* cen = ix.codebook + (static_cast<size_t>(m) * 256u + c) * SUB;
    float cv[SUB];
    if constexpr (SUB % 4 == 0) {
#pragma unroll
      for (int t = 0; t < SUB / 4; ++t) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(cen) + t);
        cv[4 * t] = v.x; cv[4 * t + 1] = v.y; cv[4 * t + 2] = v.z; cv[4 * t + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int t = 0; t < SUB; ++t) cv[t] = __ldg(cen + t);
    }
#pragma unroll
    for (int j = 0; j < SUB; ++j) {
      const int d = m * SUB + j;
      uint32_t r;
      if constexpr (RBITS == 8) r = (rw[d >> 2] >> (8 * (d & 3))) & 255u;
      else r = (rw[d >> 3] >> (4 * (d & 7))) & 15u;
      const float x = fadd(fadd(cv[j], fmul(u8f(r), qp.x)), qp.y);
      const float dq = fsub(q[d], x);
      acc = fadd(acc, fmul(dq, dq));
    }
  }
  *out_dist = acc;
  return isfinite(acc);
}

// The same, loading the candidate's rows from global memory.
template <int M, int SUB, int RBITS>
__device__ __forceinline__ bool pq_residual_fixed(const PqIndexView& ix, const float* __restrict__ q, int32_t id,
                                                  float* out_dist) {
  constexpr int DIM = M * SUB;
  constexpr int RCB = RBITS == 8 ? DIM : DIM / 2;
  constexpr int CW = (M + 3) / 4;
  constexpr int RW = RCB / 4;
  uint32_t cw[CW];
  const uint8_t* crow = ix.codes + static_cast<size_t>(id) * M;
  if constexpr (M % 16 == 0) {
#pragma unroll
    for (int i = 0; i < M / 16; ++i) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(crow) + i);
      cw[4 * i] = v.x; cw[4 * i + 1] = v.y; cw[4 * i + 2] = v.z; cw[4 * i + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < CW; ++i) cw[i] = __ldg(reinterpret_cast<const uint32_t*>(crow) + i);
  }
  uint32_t rw[RW];
  const uint8_t* res = pq_residual_row(ix, id);
  if constexpr (RCB % 16 == 0) {
#pragma unroll
    for (int i = 0; i < RCB / 16; ++i) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(res) + i);
      rw[4 * i] = v.x; rw[4 * i + 1] = v.y; rw[4 * i + 2] = v.z; rw[4 * i + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < RW; ++i) rw[i] = __ldg(reinterpret_cast<const uint32_t*>(res) + i);
  }
  const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
  return pq_residual_words<M, SUB, RBITS>(ix, q, cw, rw, qp, out_dist);
}

// ---------------------------------------------------------------------------
// Final refine of the first `count` pool entries (refine_impl with the PQ
// residual decode provider): FP32 decode ((c + code*s) + z), FP64 sum of
// squared differences in dimension order, sort by (distance, id), keep k.
// With `decoded` (the [n][dim] rows of the same decode, NaN rows for
// rejected qparams; dim % 4 == 0) the decode is read instead of recomputed:
// the same FP32 values, the same failures.
static __device__ void pq_refine_warp(const PqIndexView& ix, const float* q, const uint64_t* list,
                               int count, int k, double* sd, int32_t* si, int lane,
                               int32_t* out_ids, float* out_dists, int32_t* out_count,
                               int32_t* status, const float* decoded = nullptr, bool error4 = false) {
  int np2 = 1;
  while (np2 < count) np2 <<= 1;
  bool bad = false;
  for (int i = lane; i < np2; i += kWarp) {
    // mode ERROR4: the storage row's third-level term on top of the decode
    const int32_t row = i < count ? key_id(list[i]) : 0;
    const uint8_t* e4c = error4 && i < count ? error4_row(ix.e4, row) : nullptr;
    const float2 e4q = e4c ? __ldg(reinterpret_cast<const float2*>(ix.e4.qparams) + row) : make_float2(0.f, 0.f);
    if (i < count && decoded) {
      const int32_t id = key_id(list[i]);
      const float4* x4 = reinterpret_cast<const float4*>(decoded + static_cast<size_t>(id) * ix.dim);
      double dist = 0.0;
      for (int t = 0; t < ix.dim / 4; ++t) {
        const float4 x = __ldg(x4 + t);
        float xv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (e4c) xv[u] = error4_add(xv[u], e4c, e4q, 4 * t + u);
          if (!isfinite(xv[u])) bad = true;
          const double delta = __dsub_rn(static_cast<double>(q[4 * t + u]), static_cast<double>(xv[u]));
          dist = __dadd_rn(dist, __dmul_rn(delta, delta));
        }
      }
      if (!isfinite(dist) || dist >= 3.4028234663852886e38) bad = true;
      sd[i] = dist;
      si[i] = id;
    } else if (i < count) {
      const int32_t id = key_id(list[i]);
      const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
      const uint8_t* code = ix.codes + static_cast<size_t>(id) * ix.code_bytes;
      const uint8_t* res = pq_residual_row(ix, id);
      double dist = 0.0;
      if (!isfinite(qp.x) || !(qp.x > 0.0f) || !isfinite(qp.y)) bad = true;
      int dim = 0;
      for (int m = 0; m < ix.m; ++m) {
        const int c = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
        const float* cen = ix.codebook + (static_cast<size_t>(m) * ix.ks + c) * ix.subdim;
        for (int j = 0; j < ix.subdim; ++j, ++dim) {
          const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, dim))
                                                   : static_cast<uint32_t>(__ldg(res + dim));
          float x = fadd(fadd(__ldg(cen + j), fmul(u8f(r), qp.x)), qp.y);
          if (e4c) x = error4_add(x, e4c, e4q, dim);
          if (!isfinite(x)) bad = true;
          const double delta = __dsub_rn(static_cast<double>(q[dim]), static_cast<double>(x));
          dist = __dadd_rn(dist, __dmul_rn(delta, delta));
        }
      }
      if (!isfinite(dist) || dist >= 3.4028234663852886e38) bad = true;
      sd[i] = dist;
      si[i] = id;
    } else {
      sd[i] = __longlong_as_double(0x7ff0000000000000ll);  // +inf pads sort last
      si[i] = 0x7fffffff;
    }
  }
  if (__any_sync(kFullMask, bad)) {
    if (lane == 0) *status = kStatusNumeric;
    return;
  }
  __syncwarp();
  // bitonic sort of (distance, id) pairs in shared memory
  for (int kk = 2; kk <= np2; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < np2; i += kWarp) {
        const int p = i ^ j;
        if (p > i) {
          const bool up = (i & kk) == 0;
          const double a = sd[i], b = sd[p];
          const int32_t ia = si[i], ib = si[p];
          const bool a_gt = (a > b) || (a == b && ia > ib);
          if (up == a_gt) {
            sd[i] = b; sd[p] = a; si[i] = ib; si[p] = ia;
          }
        }
      }
      __syncwarp();
    }
  }
  const int outn = count < k ? count : k;
  for (int i = lane; i < outn; i += kWarp) {
    out_ids[i] = si[i];
    out_dists[i] = static_cast<float>(sd[i]);
  }
  if (lane == 0) *out_count = outn;
}

// ---------------------------------------------------------------------------

template <int PER>
__device__ __forceinline__ int merge_batch(uint64_t* list, int size, int cap, uint64_t* stage,
                                           uint64_t (&v)[PER], int nb, int lane) {
  // stage the sorted batch so list elements can rank against it
#pragma unroll
  for (int r = 0; r < PER; ++r) stage[lane + 32 * r] = v[r];
  __syncwarp();
  int bpos[PER];
  int min_ins = cap;
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int e = lane + 32 * r;
    bpos[r] = e < nb ? e + count_less(list, size, v[r]) : cap;
    min_ins = min(min_ins, bpos[r]);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) min_ins = min(min_ins, __shfl_xor_sync(kFullMask, min_ins, off));
  // shift list elements right, highest chunk first (new position >= old)
  const int first_chunk = min_ins >> 5;
  for (int t = (size - 1) >> 5; t >= first_chunk; --t) {
    const int i = 32 * t + lane;
    uint64_t key = 0;
    int pos = cap;
    if (i < size) {
      key = list[i];
      pos = i + count_less(stage, nb, key);
    }
    __syncwarp();
    if (i < size && pos < cap && pos != i) list[pos] = key;
    __syncwarp();
  }
#pragma unroll
  for (int r = 0; r < PER; ++r)
    if (bpos[r] < cap) list[bpos[r]] = v[r];
  __syncwarp();
  return min_ins;
}

template <int M, int SUB, int RBITS>
__device__ __forceinline__ bool score_one(const PqIndexView& ix, const float* __restrict__ q, int32_t id,
                                          bool correction, float* adc, float* dist) {
  if constexpr (M == 0) return pq_score(ix, q, id, correction, adc, dist);
  else return pq_score_fixed<M, SUB, RBITS>(ix, q, id, correction, adc, dist);
}

// Sort the scored batch (keys in `stage`) and merge it into the list.  The
// caller may first drop keys that cannot enter (drop_non_entering): they
// would land at or beyond the list's capacity and change nothing.
template <int PER>
__device__ __forceinline__ void sort_and_merge(uint64_t* list, int* size, int cap, uint64_t* stage, int nb,
                                               int* cursor, int lane) {
  uint64_t v[PER];
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int e = lane + 32 * r;
    v[r] = e < nb ? stage[e] : kEmptyKey;
  }
  __syncwarp();
  warp_bitonic_sort<PER>(v, lane);
  const int min_ins = merge_batch<PER>(list, *size, cap, stage, v, nb, lane);
  *size = min(cap, *size + nb);
  *cursor = min(*cursor, min_ins);
}

__device__ __forceinline__ void sort_merge_any(uint64_t* list, int* size, int cap, uint64_t* stage, int nb,
                                               int* cursor, int lane) {
  if (nb <= 32) sort_and_merge<1>(list, size, cap, stage, nb, cursor, lane);
  else if (nb <= 64) sort_and_merge<2>(list, size, cap, stage, nb, cursor, lane);
  else sort_and_merge<4>(list, size, cap, stage, nb, cursor, lane);
}

// Forward declaration (defined below).
__device__ __forceinline__ int drop_non_entering(const uint64_t* list, int size, int cap, uint64_t* stage, int nb,
                                                 int lane);

// Merges the scored keys stage[0..nb) (nb <= kMaxBatch) into the sorted
// list of capacity cap: keys that cannot enter are dropped first, then the
// rest are sorted and merged.  Same list, same cursor as merging them all.
__device__ __forceinline__ void merge_scored(uint64_t* list, int* size, int cap, uint64_t* stage, int nb,
                                             int* cursor, int lane) {
  nb = drop_non_entering(list, *size, cap, stage, nb, lane);
  if (nb > 0) sort_merge_any(list, size, cap, stage, nb, cursor, lane);
}

// Keys (distance, seed id) of one row of a queries x seeds distance matrix.
struct SeedRowKeys {
  const float* row;
  const int32_t* ids;
  __device__ __forceinline__ uint64_t operator()(int e, bool* nonfinite) const {
    const float d = row[e];
    if (!isfinite(d)) {
      *nonfinite = true;
      return kEmptyKey;
    }
    return make_key(d, __ldg(ids + e));
  }
};

// Keys (rank, seed index) of one row of a queries x seeds rank matrix: the
// index, not the id, so the seed's per-seed data (norms) stays reachable.
struct SeedIndexKeys {
  const float* row;
  __device__ __forceinline__ uint64_t operator()(int e, bool* nonfinite) const {
    const float d = row[e];
    if (!isfinite(d)) {
      *nonfinite = true;
      return kEmptyKey;
    }
    return make_key(d, e);
  }
};

// Top-cap selection of n keys (key_at(e), e = 0..n-1) into the sorted list:
// keys below the list's worst accumulate in stage and are merged once up to
// kMaxBatch - 32 have gathered (or at the end), so the list is merged a few
// times instead of once per chunk.  Keys are read 8 chunks (256 keys) at a
// time with every load in flight together, so a row costs n / 256 memory
// round trips.  The result is the top-cap of all keys, as inserting them
// one by one gives.  False if a distance is non-finite.
template <class KeyAt>
__device__ __forceinline__ bool select_top(uint64_t* list, int* size, int cap, uint64_t* stage, int n,
                                           const KeyAt& key_at, int* cursor, int lane) {
  constexpr int kGroup = 8;
  int cnt = 0;
  for (int g0 = 0; g0 < n; g0 += kGroup * kWarp) {
    uint64_t k[kGroup];
    bool nonfinite = false;
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      const int e = g0 + u * kWarp + lane;
      k[u] = e < n ? key_at(e, &nonfinite) : kEmptyKey;
    }
    if (__any_sync(kFullMask, nonfinite)) return false;
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      const int e0 = g0 + u * kWarp;
      if (e0 >= n) break;
      const uint64_t thr = *size == cap ? key_cmp(list[cap - 1]) : kEmptyKey;
      const bool keep = k[u] != kEmptyKey && key_cmp(k[u]) < thr;
      const unsigned km = __ballot_sync(kFullMask, keep);
      if (keep) stage[cnt + __popc(km & ((1u << lane) - 1u))] = k[u];
      cnt += __popc(km);
      if (cnt > kMaxBatch - kWarp || e0 + kWarp >= n) {
        __syncwarp();
        if (cnt) sort_merge_any(list, size, cap, stage, cnt, cursor, lane);
        cnt = 0;
      }
    }
  }
  return true;
}

// Top-cap selection (cap <= 128) of n keys in one pass: each lane keeps the
// best 8 of its keys (e = lane, lane + 32, ...) in registers, the warp merges
// those 256 candidates into the list, and T = the list's worst key decides
// exactness: a lane whose 8th best is below T may hold more keys below T, so
// it re-reads its keys and the ones in (8th best, T) are merged as well.
// The list then holds the top-cap of all n keys, as select_top gives.
template <class KeyAt>
__device__ __forceinline__ bool select_top_lanes(uint64_t* list, int* size, int cap, uint64_t* stage, int n,
                                                 const KeyAt& key_at, int* cursor, int lane) {
  constexpr int K = 8, kGroup = 8;
  uint64_t top[K];
#pragma unroll
  for (int i = 0; i < K; ++i) top[i] = kEmptyKey;
  for (int g0 = 0; g0 < n; g0 += kGroup * kWarp) {
    uint64_t k[kGroup];
    bool nonfinite = false;
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      const int e = g0 + u * kWarp + lane;
      k[u] = e < n ? key_at(e, &nonfinite) : kEmptyKey;
    }
    if (__any_sync(kFullMask, nonfinite)) return false;
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      if (k[u] < top[K - 1]) {
        uint64_t v = k[u];
#pragma unroll
        for (int i = 0; i < K; ++i) {
          const uint64_t lo = v < top[i] ? v : top[i];
          v = v < top[i] ? top[i] : v;
          top[i] = lo;
        }
      }
    }
  }
  // the lanes' best 4, then their 5th..8th (filtered by the list's worst)
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint64_t thr = *size == cap ? key_cmp(list[cap - 1]) : kEmptyKey;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint64_t v = top[4 * h + i];
      stage[i * kWarp + lane] = v < thr ? v : kEmptyKey;
    }
    __syncwarp();
    int cnt = drop_non_entering(list, *size, cap, stage, 4 * kWarp, lane);
    // empty slots sort last and never enter: count the real keys only
    int real = 0;
    for (int e = lane; e < cnt; e += kWarp) real += stage[e] != kEmptyKey;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) real += __shfl_xor_sync(kFullMask, real, off);
    if (real) {
      // compact the real keys to the front
      int c2 = 0;
      for (int e0 = 0; e0 < cnt; e0 += kWarp) {
        const int e = e0 + lane;
        const uint64_t v = e < cnt ? stage[e] : kEmptyKey;
        const bool keep = v != kEmptyKey;
        const unsigned km = __ballot_sync(kFullMask, keep);
        __syncwarp();
        if (keep) stage[c2 + __popc(km & ((1u << lane) - 1u))] = v;
        c2 += __popc(km);
        __syncwarp();
      }
      sort_merge_any(list, size, cap, stage, c2, cursor, lane);
    }
  }
  // exactness: lanes whose 8th best is below the final worst key re-read
  const uint64_t thr = *size == cap ? key_cmp(list[cap - 1]) : kEmptyKey;
  const bool rescan = top[K - 1] != kEmptyKey && top[K - 1] < thr;
  if (__any_sync(kFullMask, rescan)) {
    int cnt = 0;
    for (int e0 = 0; e0 < n; e0 += kWarp) {
      const int e = e0 + lane;
      bool nonfinite = false;
      const uint64_t v = (rescan && e < n) ? key_at(e, &nonfinite) : kEmptyKey;
      const bool keep = v > top[K - 1] && v < thr;
      const unsigned km = __ballot_sync(kFullMask, keep);
      if (keep) stage[cnt + __popc(km & ((1u << lane) - 1u))] = v;
      cnt += __popc(km);
      if (cnt > kMaxBatch - kWarp || e0 + kWarp >= n) {
        __syncwarp();
        if (cnt) sort_merge_any(list, size, cap, stage, cnt, cursor, lane);
        cnt = 0;
      }
    }
  }
  return true;
}

// Prefetches into L2 the adjacency rows of the first `count` unexpanded
// list entries at or after position `from`: the sources the next step will
// most likely expand (a better candidate merged first only wastes the hint).
__device__ __forceinline__ void prefetch_next_rows(const PqIndexView& ix, const uint64_t* list, int size, int from,
                                                   int count, int lane) {
  const int i = from + lane;
  const bool cand = i < size && !(list[i] & kExpandedBit);
  unsigned m = __ballot_sync(kFullMask, cand);
  for (int k = 0; k < count && m; ++k) {
    const int b = __ffs(m) - 1;
    m &= m - 1;
    if (lane == b) {
      const char* row = reinterpret_cast<const char*>(ix.graph + static_cast<size_t>(key_id(list[i])) * ix.degree);
      const int bytes = ix.degree * 4;
      for (int off = 0; off < bytes + 127; off += 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(row + (off < bytes ? off : bytes - 1)));
    }
  }
}

// Per-CTA Bloom filter of the entry seeds in shared memory (two hashes).  It
// has no false negatives, so a miss proves an id is not a seed and skips the
// dependent global read of the seed bitmap on the claim path; a hit is
// settled by the bitmap.  Built by every thread of the CTA before any warp
// starts a query.
__device__ __forceinline__ int filter_shift(int bits) { return 33 - __ffs(bits); }   // 32 - log2(bits)

__device__ __forceinline__ void seed_filter_build(uint32_t* f, int bits, const int32_t* __restrict__ seeds, int n) {
  for (int i = threadIdx.x; i < (bits >> 5); i += blockDim.x) f[i] = 0u;
  __syncthreads();
  const int shift = filter_shift(bits);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t u = static_cast<uint32_t>(__ldg(seeds + i));
    const uint32_t h1 = (u * 0x9E3779B1u) >> shift, h2 = hash_id(u) & static_cast<uint32_t>(bits - 1);
    atomicOr(f + (h1 >> 5), 1u << (h1 & 31));
    atomicOr(f + (h2 >> 5), 1u << (h2 & 31));
  }
  __syncthreads();
}

__device__ __forceinline__ bool seed_filter_maybe(const uint32_t* f, int bits, uint32_t u) {
  if (!bits) return true;
  const uint32_t h1 = (u * 0x9E3779B1u) >> filter_shift(bits), h2 = hash_id(u) & static_cast<uint32_t>(bits - 1);
  return ((f[h1 >> 5] >> (h1 & 31)) & (f[h2 >> 5] >> (h2 & 31)) & 1u) != 0u;
}

// Whether every LUT entry of this query is provably finite and no ADC sum
// can overflow, without building the LUT.  With every q_j and codebook entry
// finite, |fl(q - c)| <= (|q| + |c|)(1 + 2^-24), so an entry (a sequential
// sum of subdim squares) is at most 1.0001 * subdim * (max|q| + max|c|)^2;
// when that is at most FLT_MAX / (2 m) the reference's LUT and ADC checks
// cannot fail.  Otherwise the caller builds the LUT and checks it.
__device__ __forceinline__ bool lut_provably_safe(const PqIndexView& ix, const float* q, int lane) {
  float qmax = 0.0f;
  bool bad = false;
  for (int d = lane; d < ix.dim; d += kWarp) {
    const float v = q[d];
    bad |= !isfinite(v);
    qmax = fmaxf(qmax, fabsf(v));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) qmax = fmaxf(qmax, __shfl_xor_sync(kFullMask, qmax, off));
  if (__any_sync(kFullMask, bad)) return false;
  const double t = static_cast<double>(qmax) + static_cast<double>(ix.codebook_absmax);
  return 1.0001 * ix.subdim * t * t <= 3.4028234663852886e38 / (2.0 * ix.m);
}

// Drops from stage[0..nb) the keys that cannot enter a full list (not below
// its worst key), compacting the rest in order.  Returns the new count.
__device__ __forceinline__ int drop_non_entering(const uint64_t* list, int size, int cap, uint64_t* stage, int nb,
                                                 int lane) {
  if (size < cap) return nb;
  const uint64_t thr = key_cmp(list[cap - 1]);
  int cnt = 0;
  for (int e0 = 0; e0 < nb; e0 += kWarp) {
    const int e = e0 + lane;
    const uint64_t k = e < nb ? stage[e] : kEmptyKey;
    const bool keep = e < nb && key_cmp(k) < thr;
    const unsigned km = __ballot_sync(kFullMask, keep);
    __syncwarp();
    if (keep) stage[cnt + __popc(km & ((1u << lane) - 1u))] = k;
    cnt += __popc(km);
    __syncwarp();
  }
  return cnt;
}

// Writes one finished query's outputs: the sorted pool (optional), the
// statistics {scored, corrected, expanded, dedup}, and the top-k, either
// straight from the pool or through the fused final refine.
__device__ __forceinline__ void pq_finish_query(const PqSearchArgs& a, const float* q, const uint64_t* list,
                                                int size, int qi, int lane, uint8_t* base,
                                                unsigned long long scored, unsigned long long corrected,
                                                unsigned long long expanded, unsigned long long dedup,
                                                const float* decoded = nullptr) {
  const PqIndexView& ix = a.ix;
  int32_t* status = a.status + qi;
  if (a.pool_ids) {
    const int pc = min(size, a.pool_stride);  // pool_stride > 0 when pool_ids is set
    for (int i = lane; i < pc; i += kWarp) {
      const uint64_t k = list[i];
      a.pool_ids[static_cast<size_t>(qi) * a.pool_stride + i] = key_id(k);
      a.pool_dists[static_cast<size_t>(qi) * a.pool_stride + i] = key_dist(k);
    }
    if (lane == 0) a.pool_counts[qi] = pc;
  }
  if (lane == 0 && a.stats) {
    unsigned long long* s = a.stats + static_cast<size_t>(qi) * 4;
    s[0] = scored;
    s[1] = corrected;
    s[2] = expanded;
    s[3] = dedup;
  }
  if (a.out_ids) {
    const int k = min(a.top_ks ? a.top_ks[qi] : a.top_k, a.out_stride);
    const int budget = a.refine_budget;
    int32_t* oi = a.out_ids + static_cast<size_t>(qi) * a.out_stride;
    float* od = a.out_dists + static_cast<size_t>(qi) * a.out_stride;
    if (budget > 0) {
      const int cnt = min(size, budget);
      // refine scratch reuses the batch/stage area and the tail of the warp
      // slice; it is sized for max refine budget by the host.
      double* sd = reinterpret_cast<double*>(base + a.smem_refine_offset);
      int32_t* si = reinterpret_cast<int32_t*>(sd + a.refine_capacity);
      int32_t rs = kStatusOk;
      pq_refine_warp(ix, q, list, cnt, k, sd, si, lane, oi, od, a.out_counts + qi, &rs, decoded,
                     a.third_residual != 0);
      rs = __shfl_sync(kFullMask, rs, 0);
      if (rs != kStatusOk && lane == 0) *status = rs;
    } else {
      const int outn = min(size, k);
      for (int i = lane; i < outn; i += kWarp) {
        const uint64_t kk = list[i];
        oi[i] = key_id(kk);
        od[i] = key_dist(kk);
      }
      if (lane == 0) a.out_counts[qi] = outn;
    }
  }
}

}  // namespace rover
