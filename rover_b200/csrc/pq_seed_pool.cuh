// pq_seed_pool.cuh -- exact seed pool of a query from TF32-ranked seeds
// (pq_seed_rank_kernel + pq_seed_topm_kernel), verified with exact
// sequential distances: shared by the exact decoded search (pq_decoded.cu)
// and the batched search (pq_batched.cu).
#pragma once

#include "pq_common.cuh"

namespace rover {

// Corrected distance of one decoded row; false if non-finite.
template <int D>
__device__ __forceinline__ bool decoded_dist(const float* __restrict__ xrow, const float* q, int dim, float* out) {
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

// ---- verified seed pool --------------------------------------------------
//
// The exact pool after the seeds is the top-L of every seed's sequential FP32
// distance d.  Instead of computing all of them, the seeds are ranked by
// A = |q|^2 + |x|^2 - 2 q.x with TF32 tensor-core dot products
// (pq_seed_rank_kernel over the seeds' decoded rows), whose error obeys
//   |A - d| <= eps = 3 * 2^-9 sqrt(|q|^2 |x|^2) + 2^-13 (|q|^2 + |x|^2 + A):
// rounding both operands to TF32 (relative 2^-11 each) moves each product by
// at most 2^-10 of its size, an FP32 accumulation of 128 products adds well
// under 2^-13, so the dot product is within 2^-9.8 |q||x| and A within twice
// that; the FP32 norms, the final combination and the sequential sum d add
// relative errors below 2^-16 of |q|^2 + |x|^2 + d.  Both terms of eps are
// 2.6x and 8x those bounds.
//
// The L seeds of smallest A are computed exactly first; the largest of those
// L distances, U, is at least the exact L-th distance, so every seed of the
// exact top-L has A - eps <= d <= U.  The remaining seeds with A - eps <= U
// are computed too, and the top-L of everything computed is the exact top-L.
// A NaN row has A = 0 (the rank clamps at zero), ranks first and fails the
// query when its exact distance is computed, as the all-seeds pass does; a
// non-finite norm or bound sends every seed to the exact computation.
__device__ __forceinline__ float seed_eps(float qn, float xn, float a) {
  return 0.005859375f * sqrtf(qn * xn) + 1.220703125e-4f * (qn + xn + a);
}

// Exact distances of cand[0..cnt) into stage, then merged into the list;
// false if one is non-finite.
template <int D>
__device__ __forceinline__ bool exact_batch(uint64_t* list, int* size, int cap, uint64_t* stage, const int32_t* cand,
                                            int cnt, const float* decoded, const float* q, int dim, int* cursor,
                                            float* umax, int lane) {
  bool bad = false;
  float mx = 0.0f;
  for (int k = lane; k < cnt; k += kWarp) {
    const int32_t id = cand[k];
    float d;
    if (!decoded_dist<D>(decoded + static_cast<size_t>(id) * dim, q, dim, &d)) bad = true;
    mx = fmaxf(mx, d);
    stage[k] = make_key(d, id);
  }
  if (__any_sync(kFullMask, bad)) return false;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFullMask, mx, off));
  *umax = mx;
  __syncwarp();
  merge_scored(list, size, cap, stage, cnt, cursor, lane);
  return true;
}

// The exact top-cap (cap <= kVerifyMaxPool) of the seeds into list; false if an
// exact distance is non-finite (the query then fails as in the all-seeds
// pass).  Keys of the first set and of the scans are (rank, seed index).
// top / next: this query's top-M ranks from pq_seed_topm_kernel (null, or a
// NaN next, when the row must be scanned here).
template <int D>
__device__ bool verified_seed_pool(uint64_t* list, int* size, int cap, uint64_t* stage, int32_t* cand,
                                   const PqDecodedArgs& b, const float* arow, const uint64_t* top, float next,
                                   const float* q, int dim, int* cursor, int lane) {
  const int n = b.n_seeds;
  float qn = 0.0f;
  for (int t = lane; t < dim; t += kWarp) qn += q[t] * q[t];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) qn += __shfl_xor_sync(kFullMask, qn, off);
  float unused;
  // the cap seeds of smallest rank, computed exactly: their largest distance U
  bool have_top = top != nullptr && next == next;
  int s1 = 0;
  uint64_t last = 0;
  bool all = !(qn < 1e37f);
  if (have_top) {
    s1 = min(cap, n);
    last = key_cmp(top[s1 - 1]);
  } else if (!all && cap > kMaxBatch) {
    all = true;   // no top-M list for a pool wider than one batch: compute every seed
  } else if (!all) {
    if (select_top_lanes(list, size, cap, stage, n, SeedIndexKeys{arow}, cursor, lane)) {
      s1 = *size;
      last = key_cmp(list[s1 - 1]);
      for (int k = lane; k < s1; k += kWarp) cand[k] = __ldg(b.seed_ids + key_id(list[k]));
    } else {
      all = true;   // a non-finite rank: compute every seed
    }
  }
  __syncwarp();
  *size = 0;
  *cursor = 0;
  float U = 0.0f;
  if (have_top) {
    // the first set, kMaxBatch seeds at a time; U is the largest distance
    for (int c0 = 0; c0 < s1; c0 += kMaxBatch) {
      const int cn = min(kMaxBatch, s1 - c0);
      for (int k = lane; k < cn; k += kWarp) cand[k] = __ldg(b.seed_ids + key_id(top[c0 + k]));
      __syncwarp();
      float u = 0.0f;
      if (!exact_batch<D>(list, size, cap, stage, cand, cn, b.decoded, q, dim, cursor, &u, lane)) return false;
      U = fmaxf(U, u);
      __syncwarp();
    }
  } else if (s1 > 0 && !exact_batch<D>(list, size, cap, stage, cand, s1, b.decoded, q, dim, cursor, &U, lane)) {
    return false;
  }
  if (!all && s1 < cap) return true;   // every seed is in
  // With xmax the largest seed norm, A - eps <= U implies A <= T: one
  // comparison rules out almost every other seed; the few that pass take the
  // exact test.  A non-finite T computes every seed.
  const float xmax = b.seed_norm_max;
  const float K = 0.005859375f * sqrtf(qn * xmax) + 1.220703125e-4f * (qn + xmax);
  float T = (U + K) / (1.0f - 1.220703125e-4f);
  T = T * 1.0000005f;
  all = all || !(T < 1e37f);
  const float a_last = key_dist(last);
  const int e_last = key_id(last);
  int cnt = 0;
  if (have_top && !all) {
    const int m = b.top_m;
    // the listed seeds past the first set; every unlisted seed has rank >=
    // next, which rules all of them out when next (1 - 2^-13) - K > U
    const bool listed_only = n <= m || next * (1.0f - 1.220703125e-4f) * 0.9999995f - K > U;
    if (listed_only) {
      const int lim = min(m, n);
      for (int i0 = s1; i0 < lim; i0 += kWarp) {
        const int i = i0 + lane;
        bool c = false;
        int32_t id = 0;
        float a = 0.0f;
        if (i < lim) {
          const uint64_t k = top[i];
          a = key_dist(k);
          if (a <= T) {
            const int e = key_id(k);
            const float xn = __ldg(b.seed_norms + e);
            const float lo = a - seed_eps(qn, xn, a);
            c = !(lo < 1e37f && xn < 1e37f) || lo <= U;
            id = __ldg(b.seed_ids + e);
          }
        }
        const unsigned m_ = __ballot_sync(kFullMask, c);
        if (c) cand[cnt + __popc(m_ & ((1u << lane) - 1u))] = id;
        cnt += __popc(m_);
        if (cnt > kMaxBatch - kWarp) {
          __syncwarp();
          if (!exact_batch<D>(list, size, cap, stage, cand, cnt, b.decoded, q, dim, cursor, &unused, lane)) return false;
          cnt = 0;
        }
        if (!__any_sync(kFullMask, i < lim && a <= T)) break;   // ascending: the rest exceed T
      }
      __syncwarp();
      if (cnt > 0 && !exact_batch<D>(list, size, cap, stage, cand, cnt, b.decoded, q, dim, cursor, &unused, lane))
        return false;
      return true;
    }
  }
  // the row scan: every seed outside the first set ((rank, index) > last)
  // that the bound cannot rule out (every one of them when `all`); the row
  // is read as float4 (its stride is a multiple of 4), 512 seeds per round
  constexpr int kGroup = 4;
  const float4* arow4 = reinterpret_cast<const float4*>(arow);
  for (int g0 = 0; g0 < n; g0 += kGroup * kWarp * 4) {
    float4 av4[kGroup];
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      const int v = g0 / 4 + u * kWarp + lane;
      av4[u] = 4 * v < n ? arow4[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      const float aj[4] = {av4[u].x, av4[u].y, av4[u].z, av4[u].w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int e = g0 + (u * kWarp + lane) * 4 + j;
        bool c = false;
        int32_t id = 0;
        const float a = aj[j];
        if (e < n) {
          if (all) {
            c = s1 == 0 || a > a_last || (a == a_last && e > e_last) || !(a == a);
          } else if (a <= T && (a > a_last || (a == a_last && e > e_last))) {
            const float xn = __ldg(b.seed_norms + e);
            const float lo = a - seed_eps(qn, xn, a);
            c = !(lo < 1e37f && xn < 1e37f) || lo <= U;
          }
          if (c) id = __ldg(b.seed_ids + e);
        }
        const unsigned m_ = __ballot_sync(kFullMask, c);
        if (c) cand[cnt + __popc(m_ & ((1u << lane) - 1u))] = id;
        cnt += __popc(m_);
        if (cnt > kMaxBatch - kWarp) {
          __syncwarp();
          if (!exact_batch<D>(list, size, cap, stage, cand, cnt, b.decoded, q, dim, cursor, &unused, lane)) return false;
          cnt = 0;
        }
      }
    }
  }
  __syncwarp();
  if (cnt > 0 && !exact_batch<D>(list, size, cap, stage, cand, cnt, b.decoded, q, dim, cursor, &unused, lane))
    return false;
  return true;
}

}  // namespace rover
