// pq_decoded.cu -- PQ beam search with the ONLINE residual policy over
// decoded rows, on sm_100a.
//
// Same search as pq_search.cu (retrieval_pure_pq_search_scalar_with_policy,
// src/dsp_demo/retrieval_sqmd_pure_pq.c:793-969, with
// retrieval_pq_residual_query_evaluate, retrieval_pq_residual.c:983, as the
// distance policy), restructured around two facts:
//
// 1. The corrected distance of a candidate is sum_j (q_j - x_j)^2 in
//    dimension order, with x_j = (c_j + code_j * s) + z rounded per step.  x
//    does not depend on the query, so pq_decode_kernel writes it once per
//    index (FP32, n x dim).  A candidate then costs one 4*dim-byte row and
//    three FP32 operations per dimension instead of about eight.  A vector
//    whose qparams the reference rejects gets a NaN row: its distance is
//    non-finite and the query fails exactly where the reference's would.
//    The ADC distance only decides failure (non-finite ADC fails the query);
//    when every LUT entry is at most FLT_MAX / (2 m) no ADC sum can overflow,
//    so the kernel computes ADC only for queries whose LUT is that large.
//
// 2. The entry seeds (graph entry, then the LCG of pure_pq_make_seed_ids,
//    src/dsp_demo/retrieval_rpc_demo_pure_pq.c:192-208) are identical for
//    every query.  The host draws them once; pq_seed_dists_kernel computes
//    all queries x all seeds in one tiled pass (same per-pair operation
//    order); each search warp then builds its initial pool as the top-L of
//    its row under (distance, id), which is the state the reference's pool
//    reaches after inserting the seeds one by one.
//
// Visited ids: seeds are marked in a bitmap shared by all queries; the ids an
// expansion claims go into a per-warp open-addressing table in shared memory.
// A query whose expansions claim more than half that table moves its entries
// into its global generation-tagged table and continues there.

#include <cfloat>

#include "pq_common.cuh"
#include "pq_seed_pool.cuh"

namespace rover {

constexpr uint32_t kEmptySlot = 0xffffffffu;

// ---------------------------------------------------------------------------
// Decoded rows: one thread per (vector, dimension).
__global__ void pq_decode_kernel(PqIndexView ix, float* __restrict__ out) {
  const size_t total = static_cast<size_t>(ix.n) * ix.dim;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int32_t v = static_cast<int32_t>(t / ix.dim);
    const int d = static_cast<int>(t - static_cast<size_t>(v) * ix.dim);
    const int m = d / ix.subdim;
    const int j = d - m * ix.subdim;
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + v);
    const uint8_t* code = ix.codes + static_cast<size_t>(v) * ix.code_bytes;
    const int c = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
    const float cj = __ldg(ix.codebook + (static_cast<size_t>(m) * ix.ks + c) * ix.subdim + j);
    const uint8_t* res = pq_residual_row(ix, v);
    const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, d))
                                             : static_cast<uint32_t>(__ldg(res + d));
    const bool bad = !isfinite(qp.x) || !isfinite(qp.y) || !(qp.x > 0.0f);
    out[t] = bad ? __int_as_float(0x7fc00000) : fadd(fadd(cj, fmul(u8f(r), qp.x)), qp.y);
  }
}

void launch_pq_decode(const PqIndexView& ix, float* decoded, cudaStream_t s) {
  const size_t total = static_cast<size_t>(ix.n) * ix.dim;
  const int threads = 256;
  const int blocks = static_cast<int>(std::min<size_t>((total + threads - 1) / threads, 148ull * 64));
  pq_decode_kernel<<<blocks, threads, 0, s>>>(ix, decoded);
}

// ---------------------------------------------------------------------------
// All queries x all seeds: out[q][u] = sum_d (Q[q][d] - X[seed u][d])^2, each
// pair summed sequentially in dimension order like the reference's
// residual evaluation.  64 x 64 tile per CTA, 4 x 4 pairs per thread,
// dimensions staged 32 at a time (transposed) in shared memory.
constexpr int kSdTile = 64;
constexpr int kSdK = 32;

__global__ void __launch_bounds__(256) pq_seed_dists_kernel(const float* __restrict__ queries, int q_begin,
                                                            int q_end, int dim, const float* __restrict__ decoded,
                                                            const int32_t* __restrict__ seed_ids, int n_seeds,
                                                            float* __restrict__ out) {
  __shared__ __align__(16) float qs[kSdK][kSdTile + 4];
  __shared__ __align__(16) float xs[kSdK][kSdTile + 4];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int u0 = blockIdx.x * kSdTile;
  const int q0 = q_begin + blockIdx.y * kSdTile;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  // rows this thread stages (two per operand per chunk)
  const float* qrow[2];
  const float* xrow[2];
  int srow[2], scol[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int idx = tid + 256 * i;
    srow[i] = idx >> 3;
    scol[i] = (idx & 7) * 4;
    const int qq = q0 + srow[i];
    const int uu = u0 + srow[i];
    qrow[i] = qq < q_end ? queries + static_cast<size_t>(qq) * dim : nullptr;
    xrow[i] = uu < n_seeds ? decoded + static_cast<size_t>(__ldg(seed_ids + uu)) * dim : nullptr;
  }
  for (int k0 = 0; k0 < dim; k0 += kSdK) {
    const int kc = min(kSdK, dim - k0);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = scol[i];
      if (c < kc) {
        float4 qv = make_float4(0.f, 0.f, 0.f, 0.f), xv = qv;
        if (qrow[i]) qv = __ldg(reinterpret_cast<const float4*>(qrow[i] + k0 + c));
        if (xrow[i]) xv = __ldg(reinterpret_cast<const float4*>(xrow[i] + k0 + c));
        const int r = srow[i];
        qs[c][r] = qv.x; qs[c + 1][r] = qv.y; qs[c + 2][r] = qv.z; qs[c + 3][r] = qv.w;
        xs[c][r] = xv.x; xs[c + 1][r] = xv.y; xs[c + 2][r] = xv.z; xs[c + 3][r] = xv.w;
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kc; ++kk) {
      const float4 a = *reinterpret_cast<const float4*>(&qs[kk][ty * 4]);
      const float4 b = *reinterpret_cast<const float4*>(&xs[kk][tx * 4]);
      const float av[4] = {a.x, a.y, a.z, a.w};
      const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float dl = fsub(av[i], bv[j]);
          acc[i][j] = fadd(acc[i][j], fmul(dl, dl));
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int qq = q0 + ty * 4 + i;
    if (qq >= q_end) continue;
    float* orow = out + static_cast<size_t>(qq - q_begin) * n_seeds;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int uu = u0 + tx * 4 + j;
      if (uu < n_seeds) orow[uu] = acc[i][j];
    }
  }
}

void launch_pq_seed_dists(const float* queries, int q_begin, int q_end, int dim, const float* decoded,
                          const int32_t* seed_ids, int n_seeds, float* out, cudaStream_t s) {
  const dim3 grid((n_seeds + kSdTile - 1) / kSdTile, (q_end - q_begin + kSdTile - 1) / kSdTile);
  pq_seed_dists_kernel<<<grid, 256, 0, s>>>(queries, q_begin, q_end, dim, decoded, seed_ids, n_seeds, out);
}

// ---------------------------------------------------------------------------
// Seed reconstructions for ranking: x~[u] = the PQ reconstruction of seed u
// (its centroids, no residual) and |x~[u]|^2.
__global__ void pq_seed_recon_kernel(PqIndexView ix, const int32_t* __restrict__ seed_ids, int n_seeds,
                                     float* __restrict__ rows, float* __restrict__ norms) {
  const int u = blockIdx.x;
  if (u >= n_seeds) return;
  const int32_t id = seed_ids[u];
  const uint8_t* code = ix.codes + static_cast<size_t>(id) * ix.code_bytes;
  float sq = 0.0f;
  for (int d = threadIdx.x; d < ix.dim; d += blockDim.x) {
    const int m = d / ix.subdim;
    const int c = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
    const float v = __ldg(ix.codebook + (static_cast<size_t>(m) * ix.ks + c) * ix.subdim + (d - m * ix.subdim));
    rows[static_cast<size_t>(u) * ix.dim + d] = v;
    sq += v * v;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(kFullMask, sq, off);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < static_cast<int>((blockDim.x + 31) / 32); ++w) t += part[w];
    norms[u] = t;
  }
}

__global__ void pq_seed_gather_kernel(const float* __restrict__ decoded, int dim, const int32_t* __restrict__ seed_ids,
                                      int n_seeds, float* __restrict__ rows, float* __restrict__ norms) {
  const int u = blockIdx.x;
  if (u >= n_seeds) return;
  const float* src = decoded + static_cast<size_t>(seed_ids[u]) * dim;
  float sq = 0.0f;
  for (int d = threadIdx.x; d < dim; d += blockDim.x) {
    const float v = __ldg(src + d);
    rows[static_cast<size_t>(u) * dim + d] = v;
    sq += v * v;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(kFullMask, sq, off);
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < static_cast<int>((blockDim.x + 31) / 32); ++w) t += part[w];
    norms[u] = t;
  }
}

// One CTA per row.  The ranks are non-negative floats (the rank kernel
// clamps at zero), so their bit patterns order as unsigned integers.  A first
// pass finds the row's smallest and largest bits; every rank shares their
// common leading bits, so one 256-bin histogram of the next 8 bits finds the
// bin b that holds the (m+1)-th smallest rank.  Every rank up to the end of
// bin b is gathered as a key (rank, seed index) and sorted; the first m are
// the row's m smallest, and the (m+1)-th is among them.  When bin b holds
// too many ranks to gather, a radix select of 8 bits per pass (MSB first)
// finds the (m+1)-th rank t exactly and the ranks <= t are gathered instead.
// A non-finite rank, or more than kTopGather ranks <= t, marks the row for a
// scan by the search kernel (empty keys, NaN next).
constexpr int kTopThreads = 128;
constexpr int kTopGather = 2048;   // gathered keys held in shared memory

__global__ void __launch_bounds__(kTopThreads) pq_seed_topm_kernel(const float* __restrict__ rank, int stride,
                                                                   int n_seeds, int rows, int m,
                                                                   uint64_t* __restrict__ keys,
                                                                   float* __restrict__ next) {
  __shared__ unsigned hist[256];
  __shared__ unsigned s_prefix, s_mask, s_remaining, s_count, s_bin_count;
  __shared__ unsigned s_lo[kTopThreads / kWarp], s_hi[kTopThreads / kWarp];
  __shared__ uint64_t gathered[kTopGather];
  const int row = blockIdx.x;
  if (row >= rows) return;
  const float* r = rank + static_cast<size_t>(row) * stride;
  const int tid = threadIdx.x;
  // f(e, rank) over the row, 16 bytes per load when the rows allow it
  const bool v4 = (stride & 3) == 0 && (reinterpret_cast<uintptr_t>(rank) & 15u) == 0;
  // (four loads in flight per thread before any is used)
  auto each = [&](auto&& f) {
    int e0 = 0;
    if (v4) {
      const int n4 = n_seeds >> 2;
      const float4* r4 = reinterpret_cast<const float4*>(r);
      for (int i = tid; i < n4; i += 4 * kTopThreads) {
        float4 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = i + u * kTopThreads;
          x[u] = j < n4 ? __ldg(r4 + j) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = i + u * kTopThreads;
          if (j < n4) {
            f(4 * j, x[u].x);
            f(4 * j + 1, x[u].y);
            f(4 * j + 2, x[u].z);
            f(4 * j + 3, x[u].w);
          }
        }
      }
      e0 = 4 * n4;
    }
    for (int e = e0 + tid; e < n_seeds; e += kTopThreads) f(e, __ldg(r + e));
  };
  bool bad = false;
  uint32_t lo = 0xffffffffu, hi = 0u;
  each([&](int, float x) {
    bad |= !(x < 3.0e38f);
    const uint32_t v = __float_as_uint(x + 0.0f);
    lo = min(lo, v);
    hi = max(hi, v);
  });
  uint64_t* out = keys + static_cast<size_t>(row) * m;
  if (__syncthreads_or(bad)) {
    for (int i = tid; i < m; i += kTopThreads) out[i] = kEmptyKey;
    if (tid == 0) next[row] = __int_as_float(0x7fc00000);
    return;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(kFullMask, lo, off));
    hi = max(hi, __shfl_xor_sync(kFullMask, hi, off));
  }
  if ((tid & 31) == 0) { s_lo[tid >> 5] = lo; s_hi[tid >> 5] = hi; }
  __syncthreads();
  lo = s_lo[0];
  hi = s_hi[0];
#pragma unroll
  for (int w = 1; w < kTopThreads / kWarp; ++w) { lo = min(lo, s_lo[w]); hi = max(hi, s_hi[w]); }
  const int target = min(m + 1, n_seeds);   // rank (1-based) of the value to find

  // One histogram pass over bits [shift, shift + 8) of the ranks matching
  // (prefix, mask); narrows prefix / mask / remaining to the target's bin.
  auto radix_pass = [&](int shift) {
    for (int i = tid; i < 256; i += kTopThreads) hist[i] = 0u;
    __syncthreads();
    const unsigned prefix = s_prefix, mask = s_mask;
    each([&](int, float x) {
      const uint32_t v = __float_as_uint(x + 0.0f);
      if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & 255u], 1u);
    });
    __syncthreads();
    if (tid < kWarp) {
      // the bin holding the remaining-th element: lane l owns bins 8l..8l+7
      const int lane = tid;
      unsigned own[8], sum = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) { own[k] = hist[8 * lane + k]; sum += own[k]; }
      unsigned incl = sum;
#pragma unroll
      for (int off = 1; off < kWarp; off <<= 1) {
        const unsigned v = __shfl_up_sync(kFullMask, incl, off);
        if (lane >= off) incl += v;
      }
      const unsigned rem0 = s_remaining;
      const unsigned hit = __ballot_sync(kFullMask, incl >= rem0);
      const int owner = hit ? __ffs(hit) - 1 : kWarp - 1;
      if (lane == owner) {
        unsigned rem = rem0 - (incl - sum), bin = 8u * lane, in_bin = own[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) {
          if (own[k] >= rem) {
            in_bin = own[k];
            break;
          }
          rem -= own[k];
          ++bin;
        }
        s_remaining = rem;
        s_bin_count = in_bin;
        s_prefix = prefix | (bin << shift);
        s_mask = mask | (255u << shift);
      }
    }
    __syncthreads();
  };
  // Gathers every rank <= t as a key; returns how many there are.
  auto gather = [&](uint32_t t) -> int {
    if (tid == 0) s_count = 0u;
    __syncthreads();
    each([&](int e, float x) {
      const uint32_t v = __float_as_uint(x + 0.0f);
      if (v <= t) {
        const unsigned slot = atomicAdd(&s_count, 1u);
        if (slot < kTopGather) gathered[slot] = (static_cast<uint64_t>(v) << 32) | static_cast<uint32_t>(e);
      }
    });
    __syncthreads();
    return static_cast<int>(s_count);
  };

  // the 8 bits below the leading bits every rank shares
  const int common = lo == hi ? 32 : __clz(lo ^ hi);
  const int first = max(0, 24 - common);
  const unsigned top = first + 8 >= 32 ? 0u : (0xffffffffu << (first + 8));
  if (tid == 0) { s_prefix = lo & top; s_mask = top; s_remaining = static_cast<unsigned>(target); }
  __syncthreads();
  radix_pass(first);
  // narrow a crowded bin 8 bits at a time while that leaves more ranks up
  // to its end than one warp sorts in registers
  int shift = first;
  while (shift >= 8 && static_cast<int>(target - s_remaining + s_bin_count) > 8 * kWarp) {
    shift -= 8;
    radix_pass(shift);
  }
  int cnt = gather(s_prefix | ((1u << shift) - 1u));   // every rank up to the end of the target's bin
  if (cnt > kTopGather) {
    // a crowded bin: the exact (m+1)-th rank, 8 bits per pass from the top
    if (tid == 0) { s_prefix = 0u; s_mask = 0u; s_remaining = static_cast<unsigned>(target); }
    __syncthreads();
    for (int shift = 24; shift >= 0; shift -= 8) radix_pass(shift);
    cnt = gather(s_prefix);
  }
  if (cnt > kTopGather) {   // a flood of equal ranks: let the search kernel scan the row
    for (int i = tid; i < m; i += kTopThreads) out[i] = kEmptyKey;
    if (tid == 0) next[row] = __int_as_float(0x7fc00000);
    return;
  }
  if (cnt <= 8 * kWarp) {
    // one warp sorts in registers
    if (tid < kWarp) {
      uint64_t v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = tid + kWarp * r < cnt ? gathered[tid + kWarp * r] : kEmptyKey;
      warp_bitonic_sort<8>(v, tid);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = tid + kWarp * r;
        if (i < m) out[i] = i < cnt ? v[r] : kEmptyKey;
        if (i == m && n_seeds > m) next[row] = __uint_as_float(static_cast<uint32_t>(v[r] >> 32));
      }
      for (int i = 8 * kWarp + tid; i < m; i += kWarp) out[i] = kEmptyKey;
      if (tid == 0 && n_seeds <= m) next[row] = __int_as_float(0x7f800000);
    }
    return;
  }
  int np2 = 1;
  while (np2 < cnt) np2 <<= 1;
  for (int i = cnt + tid; i < np2; i += kTopThreads) gathered[i] = kEmptyKey;
  __syncthreads();
  for (int k = 2; k <= np2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < np2; i += kTopThreads) {
        const int p = i ^ j;
        if (p > i) {
          const uint64_t x = gathered[i], y = gathered[p];
          if (((i & k) == 0) == (x > y)) { gathered[i] = y; gathered[p] = x; }
        }
      }
      __syncthreads();
    }
  for (int i = tid; i < m; i += kTopThreads) out[i] = i < cnt ? gathered[i] : kEmptyKey;
  if (tid == 0) next[row] = n_seeds > m ? __uint_as_float(static_cast<uint32_t>(gathered[m] >> 32)) : __int_as_float(0x7f800000);
}

void launch_pq_seed_topm(const float* rank, int stride, int n_seeds, int rows, int m, uint64_t* keys, float* next,
                         cudaStream_t s) {
  if (rows <= 0 || m <= 0) return;
  pq_seed_topm_kernel<<<rows, kTopThreads, 0, s>>>(rank, stride, n_seeds, rows, m, keys, next);
}

void launch_pq_seed_gather(const float* decoded, int dim, const int32_t* seed_ids, int n_seeds, float* rows,
                           float* norms, cudaStream_t s) {
  pq_seed_gather_kernel<<<n_seeds, 128, 0, s>>>(decoded, dim, seed_ids, n_seeds, rows, norms);
}

void launch_pq_seed_recon(const PqIndexView& ix, const int32_t* seed_ids, int n_seeds, float* rows, float* norms,
                          cudaStream_t s) {
  pq_seed_recon_kernel<<<n_seeds, 128, 0, s>>>(ix, seed_ids, n_seeds, rows, norms);
}

// All queries x all seeds, quantized distance for ranking, on the tensor
// cores: out[q][u] = |q|^2 + |x~_u|^2 - 2 q . x~_u with the dot products as
// TF32 mma.sync m16n8k8 tiles (FP32 accumulation).  It is not the
// reference's ADC sum (different order and TF32 operands); the gated search
// only ranks seeds with it, and corrects the ones it keeps exactly.
constexpr int kRkTile = 64;
constexpr int kRkK = 32;

__device__ __forceinline__ uint32_t to_tf32(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const uint32_t* p) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

// Operands are staged in shared memory already rounded to TF32, two K
// chunks deep: the next chunk's global loads are in flight while the tensor
// cores work on the current one.  Thread tid stages rows tid / 8 + 16 j
// (j < 4), columns 4 (tid % 8) .. + 3 of every chunk, and sums those
// columns' squares of its query rows; eight lanes then add their parts.
__global__ void __launch_bounds__(128) pq_seed_rank_kernel(const float* __restrict__ queries, int q_begin, int q_end,
                                                           int dim, const float* __restrict__ rows,
                                                           const float* __restrict__ norms, int n_seeds,
                                                           float* __restrict__ out, int out_stride) {
  __shared__ __align__(16) uint32_t qs[2][kRkTile][kRkK + 4];
  __shared__ __align__(16) uint32_t xs[2][kRkTile][kRkK + 4];
  __shared__ float qn[kRkTile];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;   // this warp's 32 x 32 sub-tile
  const int q0 = q_begin + blockIdx.y * kRkTile, u0 = blockIdx.x * kRkTile;
  const int sr = tid >> 3, sc = (tid & 7) * 4;             // staging row (+16 j) and column
  constexpr int kRows = kRkTile / 16;
  float4 pq[kRows], px[kRows];
  float qsq[kRows] = {};
  auto load = [&](int k0) {
    const bool in_k = sc < min(kRkK, dim - k0);
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      const int r = sr + 16 * j;
      pq[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      px[j] = pq[j];
      if (in_k) {
        if (q0 + r < q_end) pq[j] = __ldg(reinterpret_cast<const float4*>(queries + static_cast<size_t>(q0 + r) * dim + k0 + sc));
        if (u0 + r < n_seeds) px[j] = __ldg(reinterpret_cast<const float4*>(rows + static_cast<size_t>(u0 + r) * dim + k0 + sc));
      }
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      const int r = sr + 16 * j;
      const float4 a = pq[j], b = px[j];
      qsq[j] += ((a.x * a.x + a.y * a.y) + a.z * a.z) + a.w * a.w;
      *reinterpret_cast<uint4*>(&qs[buf][r][sc]) = make_uint4(to_tf32(a.x), to_tf32(a.y), to_tf32(a.z), to_tf32(a.w));
      *reinterpret_cast<uint4*>(&xs[buf][r][sc]) = make_uint4(to_tf32(b.x), to_tf32(b.y), to_tf32(b.z), to_tf32(b.w));
    }
  };
  float acc[2][4][4] = {};
  load(0);
  store(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < dim; k0 += kRkK) {
    const bool more = k0 + kRkK < dim;
    if (more) load(k0 + kRkK);
#pragma unroll
    for (int kk = 0; kk < kRkK; kk += 8) {
      // ldmatrix x4: lanes 8i .. 8i+7 address the rows of 8 x 4-word matrix
      // i, and register i of lane l receives word l % 4 of row l / 4 of it.
      // A (rows q, words k): matrices (rows 0-7, k 0-3), (8-15, 0-3),
      // (0-7, 4-7), (8-15, 4-7) are a0..a3 of m16n8k8.  B (rows seed,
      // words k): (ni, k 0-3), (ni, 4-7) are b0, b1; two ni per load.
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
        ldsm_x4(a[mi], &qs[buf][wm + mi * 16 + (lane & 7) + 8 * ((lane >> 3) & 1)][kk + 4 * (lane >> 4)]);
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        uint32_t r4[4];
        ldsm_x4(r4, &xs[buf][wn + (2 * p + (lane >> 4)) * 8 + (lane & 7)][kk + 4 * ((lane >> 3) & 1)]);
        b[2 * p][0] = r4[0];
        b[2 * p][1] = r4[1];
        b[2 * p + 1][0] = r4[2];
        b[2 * p + 1][1] = r4[3];
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
          asm volatile(
              "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
              "{%0,%1,%2,%3};\n"
              : "+f"(acc[mi][ni][0]), "+f"(acc[mi][ni][1]), "+f"(acc[mi][ni][2]), "+f"(acc[mi][ni][3])
              : "r"(a[mi][0]), "r"(a[mi][1]), "r"(a[mi][2]), "r"(a[mi][3]), "r"(b[ni][0]), "r"(b[ni][1]));
    }
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int j = 0; j < kRows; ++j) {
    float v = qsq[j];
    v += __shfl_xor_sync(kFullMask, v, 1);
    v += __shfl_xor_sync(kFullMask, v, 2);
    v += __shfl_xor_sync(kFullMask, v, 4);
    if ((tid & 7) == 0) qn[sr + 16 * j] = v;
  }
  __syncthreads();
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = wm + mi * 16 + g + 8 * h;
      const int qq = q0 + r;
      if (qq >= q_end) continue;
      float* orow = out + static_cast<size_t>(qq - q_begin) * out_stride;
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int uu = u0 + wn + ni * 8 + 2 * t + e;
          if (uu < n_seeds) orow[uu] = fmaxf(qn[r] + __ldg(norms + uu) - 2.0f * acc[mi][ni][2 * h + e], 0.0f);
        }
    }
}

void launch_pq_seed_rank(const float* queries, int q_begin, int q_end, int dim, const float* rows, const float* norms,
                         int n_seeds, float* out, cudaStream_t s, int out_stride) {
  const dim3 grid((n_seeds + kRkTile - 1) / kRkTile, (q_end - q_begin + kRkTile - 1) / kRkTile);
  pq_seed_rank_kernel<<<grid, 128, 0, s>>>(queries, q_begin, q_end, dim, rows, norms, n_seeds, out,
                                           out_stride ? out_stride : n_seeds);
}

// ---------------------------------------------------------------------------

// Shared-memory visited insert: 1 = first visit, 0 = seen, -1 = no slot.
__device__ __forceinline__ int smem_visit(uint32_t* tab, uint32_t mask, uint32_t id) {
  uint32_t h = hash_id(id) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t prev = atomicCAS(tab + h, kEmptySlot, id);
    if (prev == kEmptySlot) return 1;
    if (prev == id) return 0;
    h = (h + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

template <int D>
__global__ void __launch_bounds__(kMaxSearchWarps * 32, 16 / kMaxSearchWarps)
pq_decoded_search_kernel(PqSearchArgs a, PqDecodedArgs b) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint32_t* seed_filter = reinterpret_cast<uint32_t*>(smem);
  uint8_t* base = smem + b.filter_bits / 8 + static_cast<size_t>(warp) * a.smem_per_warp;
  float* q = reinterpret_cast<float*>(base);
  uint64_t* list = reinterpret_cast<uint64_t*>(base + a.smem_query_bytes);
  uint64_t* stage = list + a.max_pool;
  int32_t* batch = reinterpret_cast<int32_t*>(stage + kMaxBatch);
  uint32_t* vis = reinterpret_cast<uint32_t*>(base + b.smem_vis_offset);
  const uint32_t vmask = static_cast<uint32_t>(b.vis_cap - 1);
  const int slot = blockIdx.x * (blockDim.x >> 5) + warp;   // warps per CTA: set at launch
  VisitedTable vt;
  vt.slots = a.visited + static_cast<size_t>(slot) * (a.visited_mask + 1ull);
  vt.mask = a.visited_mask;
  const PqIndexView& ix = a.ix;
  const int dim = D ? D : ix.dim;
  const float adc_bound = FLT_MAX / static_cast<float>(2 * ix.m);

  if (b.filter_bits) seed_filter_build(seed_filter, b.filter_bits, b.seed_ids, b.n_seeds);
  for (;;) {
    int item = 0;
    if (lane == 0) item = b.q_begin + static_cast<int>(atomicAdd(a.next_query, 1u));
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= b.q_end) break;
    // with an order, items index it and the seed rows cover every query
    const int qi = a.order ? __ldg(a.order + item) : item;
    const size_t seed_row_index = static_cast<size_t>(a.order ? qi : qi - b.q_begin);
    const size_t seed_row = seed_row_index * (b.seed_stride ? b.seed_stride : b.n_seeds);

    const int cap = a.pool_sizes[qi];
    int32_t* status = a.status + qi;
    const int expand = min(a.expand_count, ix.degree);
    if (cap <= 0 || cap > a.max_pool || expand <= 0 || expand > kMaxBatch || a.entry_points <= 0) {
      if (lane == 0) *status = kStatusBadParam;
      continue;
    }
    if (b.seed_err && *reinterpret_cast<const volatile int*>(b.seed_err)) {
      if (lane == 0) *status = kStatusSeedRank;
      continue;
    }
    {
      const float4* src = reinterpret_cast<const float4*>(a.queries + static_cast<size_t>(qi) * dim);
      for (int t = lane; t < dim / 4; t += kWarp) reinterpret_cast<float4*>(q)[t] = __ldg(src + t);
    }
    for (int i = lane; i < b.vis_cap; i += kWarp) vis[i] = kEmptySlot;
    __syncwarp();
    // retrieval_pq_build_lut fails the query if any LUT entry is not finite;
    // the largest entry decides whether ADC sums need checking at all.  The
    // LUT is only built when the bound cannot settle both.
    bool check_adc = false;
    if (!lut_provably_safe(ix, q, lane)) {
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
    unsigned long long scored = static_cast<unsigned long long>(b.n_seeds), expanded = 0;
    unsigned long long dedup = lane == 0 ? static_cast<unsigned long long>(b.seed_dups) : 0ull;
    int32_t st = kStatusOk;

    // ---- initial pool: top-L of the seed row under (distance, id)
    const float* drow = b.seed_dists + seed_row;
    if (b.seed_verify) {
      // the host sets seed_verify only when every pool fits kVerifyMaxPool
      if (cap > kVerifyMaxPool) st = kStatusBadParam;
      else if (!verified_seed_pool<D>(list, &size, cap, stage, batch, b, drow,
                                      b.seed_top ? b.seed_top + seed_row_index * b.top_m : nullptr,
                                      b.seed_top ? b.seed_top_next[seed_row_index] : 0.0f,
                                      q, dim, &cursor, lane))
        st = kStatusNumeric;
    } else if (!(cap <= kMaxBatch
                     ? select_top_lanes(list, &size, cap, stage, b.n_seeds, SeedRowKeys{drow, b.seed_ids}, &cursor, lane)
                     : select_top(list, &size, cap, stage, b.n_seeds, SeedRowKeys{drow, b.seed_ids}, &cursor, lane))) {
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

    // ---- expansion loop (first unexpanded list entry, as pq_search.cu)
    bool global_mode = false;
    int claimed = 0;  // ids claimed by expansions of this query
    const uint32_t load_limit = (a.visited_mask + 1u) >> 1;
    while (st == kStatusOk) {
      int pos = -1;
      for (int b0 = cursor & ~31; b0 < size; b0 += kWarp) {
        const int i = b0 + lane;
        const bool cand = i >= cursor && i < size && !(list[i] & kExpandedBit);
        const unsigned m = __ballot_sync(kFullMask, cand);
        if (m) { pos = b0 + __ffs(m) - 1; break; }
      }
      if (pos < 0) break;
      cursor = pos + 1;
      const int32_t src = key_id(list[pos]);
      prefetch_next_rows(ix, list, size, pos + 1, 1, lane);
      __syncwarp();
      if (lane == 0) list[pos] |= kExpandedBit;
      const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
      // valid-prefix rule (pure_pq_graph_row_count)
      int first_pad = expand;
      bool row_bad = false;
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
#pragma unroll
      for (int r = 0; r < kMaxBatch / kWarp; ++r) {
        const int j = r * kWarp + lane;
        if (j < expand) {
          const int32_t nid = nid_r[r];
          if (j < first_pad) row_bad |= (nid < 0 || nid >= ix.n);
          else row_bad |= (nid != -1);
        }
      }
      if (__any_sync(kFullMask, row_bad)) { st = kStatusBadRow; break; }
      // move to the global table before this row could push the shared one
      // past half load
      bool full = false;
      if (!global_mode && claimed + first_pad > b.vis_cap / 2) {
        for (int i = lane; i < b.vis_cap; i += kWarp) {
          const uint32_t id = vis[i];
          if (id != kEmptySlot && visited_insert(vt, id) < 0) full = true;
        }
        global_mode = true;
        __syncwarp();
      }
      // first visits, in row order
      int nb = 0;
#pragma unroll
      for (int r = 0; r < kMaxBatch / kWarp; ++r) {
        if (r * kWarp < first_pad) {
          const int j = r * kWarp + lane;
          int fresh = 0;
          const int32_t nid = nid_r[r];
          if (j < first_pad) {
            const uint32_t u = static_cast<uint32_t>(nid);
            if (seed_filter_maybe(seed_filter, b.filter_bits, u) && (__ldg(b.seed_bits + (u >> 5)) & (1u << (u & 31)))) {
              ++dedup;
            } else {
              const int rr = global_mode ? visited_insert(vt, u) : smem_visit(vis, vmask, u);
              full |= rr < 0;
              fresh = rr == 1;
              if (rr == 0) ++dedup;
            }
          }
          const unsigned fm = __ballot_sync(kFullMask, fresh);
          if (fresh) batch[nb + __popc(fm & ((1u << lane) - 1u))] = nid;
          nb += __popc(fm);
        }
      }
      ++expanded;
      claimed += nb;
      if (__any_sync(kFullMask, full) || (global_mode && static_cast<uint32_t>(claimed) > load_limit)) {
        st = kStatusTableFull;
        break;
      }
      __syncwarp();
      if (nb == 0) continue;
      scored += nb;
      // score: one lane per candidate, rows prefetched first
      for (int e = lane; e < nb; e += kWarp) {
        const float* xr = b.decoded + static_cast<size_t>(batch[e]) * dim;
        for (int off = 0; off < dim; off += 32) prefetch_l1(xr + off);
      }
      bool sbad = false;
      for (int e = lane; e < nb; e += kWarp) {
        const int32_t id = batch[e];
        float dist;
        if (!decoded_dist<D>(b.decoded + static_cast<size_t>(id) * dim, q, dim, &dist)) sbad = true;
        if (check_adc) {
          float adc, unused;
          if (!pq_score(ix, q, id, false, &adc, &unused)) sbad = true;
        }
        stage[e] = make_key(dist, id);
      }
      if (__any_sync(kFullMask, sbad)) { st = kStatusNumeric; break; }
      __syncwarp();
      merge_scored(list, &size, cap, stage, nb, &cursor, lane);
    }

#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dedup += __shfl_xor_sync(kFullMask, dedup, off);
    if (st != kStatusOk) {
      if (lane == 0) *status = st;
      continue;
    }
    __syncwarp();
    pq_finish_query(a, q, list, size, qi, lane, base, scored, scored, expanded, dedup, b.decoded);
    __syncwarp();
  }
}

PqDecodedFn pq_decoded_kernel_for(int dim) {
  if (dim % 4 != 0) return nullptr;
  switch (dim) {
    case 128: return pq_decoded_search_kernel<128>;
    case 96: return pq_decoded_search_kernel<96>;
    case 64: return pq_decoded_search_kernel<64>;
    default: return pq_decoded_search_kernel<0>;
  }
}

}  // namespace rover
