// distance.cu -- batched distance kernels (the standalone K1/K2/K3/K5/K6
// kernels) for scoring explicit (query, id) lists: the lane-protocol
// sessions, the score-ids entry points and the re-rank of host-supplied
// candidate lists use them.
//
//  pq_lut_kernel       retrieval_pq_build_lut      (retrieval_pq_core.c:362)
//  pq_adc_kernel       retrieval_pq_adc_ids_batch  (retrieval_pq_core.c:280-360)
//  pq_residual_kernel  retrieval_pq_residual_query_evaluate (retrieval_pq_residual.c:983)
//  sq_coarse_kernel    retrieval_compute_int8_native_distance_u8 / int4 (l1_int8_core.c:119-169)
//  sq_exact_kernel     retrieval_demo_exact_distance_residual (retrieval_rpc_demo_support.c:1397)
//  refine_kernel       refine_impl (retrieval_final_refine.c:256-292)
//
// Each query's id list is offsets[q] .. offsets[q+1] of a flat id array.

#include "pq_common.cuh"
#include "sq_split.cuh"

namespace rover {

__device__ __forceinline__ const uint8_t* residual_row(const PqIndexView& ix, int32_t id) {
  const uint32_t u = static_cast<uint32_t>(id);
  const uint32_t block = u / static_cast<uint32_t>(ix.vpb);
  return ix.residual + static_cast<size_t>(block) * 4096u +
         (u - block * static_cast<uint32_t>(ix.vpb)) * static_cast<uint32_t>(ix.rcb);
}

// ---------------------------------------------------------------------------
// Staged gathers: a warp takes 32 candidate ids at a time and streams their
// rows into its shared-memory tile with cp.async (no register staging, all
// of the tile's copies in flight at once), then each lane scores its
// candidate from shared memory.  Row strides are odd multiples of 16 bytes
// so that the 16-byte reads of 8 lanes fall in distinct bank groups.
constexpr int kStageWarps = 4;

__device__ __forceinline__ constexpr int stage_stride(int row_bytes) {
  return ((((row_bytes + 15) / 16) | 1) * 16);
}

template <int CHUNK>
__device__ __forceinline__ void cp_async_chunk(void* dst, const void* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if constexpr (CHUNK == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else if constexpr (CHUNK == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Copies rows r = 0..cnt-1 of row_bytes (a multiple of CHUNK, sources
// CHUNK-aligned) from src(r) to dst + r * stride.
template <int CHUNK, class Src>
__device__ __forceinline__ void stage_rows(uint8_t* dst, int stride, int row_bytes, int cnt, const Src& src, int lane) {
  const int per = row_bytes / CHUNK;
  for (int c = lane; c < cnt * per; c += kWarp) {
    const int r = c / per, k = c - r * per;
    cp_async_chunk<CHUNK>(dst + r * stride + k * CHUNK, src(r) + k * CHUNK);
  }
}

__global__ void pq_lut_kernel(PqIndexView ix, const float* __restrict__ queries, int nq,
                              float* __restrict__ luts, int32_t* status) {
  const int qi = blockIdx.x;
  const float* q = queries + static_cast<size_t>(qi) * ix.dim;
  const int entries = ix.m * ix.ks;
  bool bad = false;
  for (int e = threadIdx.x; e < entries; e += blockDim.x) {
    const int m = e / ix.ks;
    const float* cen = ix.codebook + static_cast<size_t>(e) * ix.subdim;
    const float* qs = q + m * ix.subdim;
    float acc = 0.0f;
    for (int j = 0; j < ix.subdim; ++j) {
      const float diff = fsub(__ldg(qs + j), __ldg(cen + j));
      acc = fadd(acc, fmul(diff, diff));
    }
    bad |= !isfinite(acc);
    luts[static_cast<size_t>(qi) * entries + e] = acc;
  }
  if (bad) status[qi] = kStatusNumeric;
}

// One CTA per query: the query's LUT is staged in shared memory, then each
// thread gathers one candidate's code row and sums its M LUT entries in
// subspace order.
__global__ void pq_adc_kernel(PqIndexView ix, const float* __restrict__ luts, int nq,
                              const int32_t* __restrict__ ids, const int64_t* __restrict__ offsets,
                              float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(16) float lut[];
  const int qi = blockIdx.y;
  const int entries = ix.m * ix.ks;
  const float* src = luts + static_cast<size_t>(qi) * entries;
  for (int e = threadIdx.x; e < entries; e += blockDim.x) lut[e] = __ldg(src + e);
  __syncthreads();
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  bool bad = false;
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = __ldg(ids + i);
    if (id < 0 || id >= ix.n) { bad = true; continue; }
    const uint8_t* code = ix.codes + static_cast<size_t>(id) * ix.code_bytes;
    float acc = 0.0f;
    if (ix.ks == 256 && (ix.code_bytes & 15) == 0) {
      for (int w = 0; w < ix.code_bytes; w += 16) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(code + w));
        const uint32_t words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int m = w + k;
          const uint32_t c = (words[k >> 2] >> (8 * (k & 3))) & 255u;
          acc = fadd(acc, lut[m * 256 + c]);
        }
      }
    } else {
      for (int m = 0; m < ix.m; ++m) {
        const int c = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
        acc = fadd(acc, lut[m * ix.ks + c]);
      }
    }
    if (!isfinite(acc)) bad = true;
    out[i] = acc;
  }
  if (bad) status[qi] = kStatusNumeric;
}

template <int M, int SUB, int RBITS>
__global__ void pq_residual_kernel(PqIndexView ix, const float* __restrict__ queries, int nq,
                                   const int32_t* __restrict__ ids,
                                   const int64_t* __restrict__ offsets, float* __restrict__ out,
                                   int32_t* status) {
  extern __shared__ __align__(16) float qs[];
  const int qi = blockIdx.y;
  for (int d = threadIdx.x; d < ix.dim; d += blockDim.x)
    qs[d] = queries[static_cast<size_t>(qi) * ix.dim + d];
  __syncthreads();
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  bool bad = false;
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = __ldg(ids + i);
    if (id < 0 || id >= ix.n) { bad = true; continue; }
    if constexpr (M > 0) {
      float acc;
      if (!pq_residual_fixed<M, SUB, RBITS>(ix, qs, id, &acc)) { bad = true; continue; }
      out[i] = acc;
    } else {
      const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
      if (!isfinite(qp.x) || !isfinite(qp.y) || !(qp.x > 0.0f)) { bad = true; continue; }
      const uint8_t* code = ix.codes + static_cast<size_t>(id) * ix.code_bytes;
      const uint8_t* res = residual_row(ix, id);
      float acc = 0.0f;
      int dim = 0;
      for (int m = 0; m < ix.m; ++m) {
        const int c = ix.ks == 16 ? nibble(code, m) : __ldg(code + m);
        const float* cen = ix.codebook + (static_cast<size_t>(m) * ix.ks + c) * ix.subdim;
        for (int j = 0; j < ix.subdim; ++j, ++dim) {
          const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, dim))
                                                   : static_cast<uint32_t>(__ldg(res + dim));
          const float x = fadd(fadd(__ldg(cen + j), fmul(u8f(r), qp.x)), qp.y);
          const float dq = fsub(qs[dim], x);
          acc = fadd(acc, fmul(dq, dq));
        }
      }
      if (!isfinite(acc)) bad = true;
      out[i] = acc;
    }
  }
  if (bad) status[qi] = kStatusNumeric;
}

// The corrected distance of kind 1 over decoded rows x = (c + code*s) + z
// (dim % 4 == 0).  Each warp takes 32 ids at a time and streams their rows
// into shared memory with cp.async (16 bytes per lane and instruction,
// every row of the tile in flight at once, no register staging), then each
// lane sums its candidate's row in dimension order, the same FP32 sequence
// as kind 1.  Rows are padded by 4 floats so the 16-byte reads of 8 lanes
// fall in distinct bank groups.
constexpr int kRescoreWarps = 4;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__global__ void __launch_bounds__(kRescoreWarps * 32) pq_rescore_kernel(int dim, int n, const float* __restrict__ decoded,
                                                                        const float* __restrict__ queries, int nq,
                                                                        const int32_t* __restrict__ ids,
                                                                        const int64_t* __restrict__ offsets,
                                                                        float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(16) float sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rs = dim + 4;
  float* qs = sm;
  float* tile = sm + dim + static_cast<size_t>(warp) * kWarp * rs;
  const int qi = blockIdx.y;
  for (int d = threadIdx.x; d < dim; d += blockDim.x) qs[d] = queries[static_cast<size_t>(qi) * dim + d];
  __syncthreads();
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  const int n4 = dim / 4;
  bool bad = false;
  for (int64_t b0 = begin + (static_cast<int64_t>(blockIdx.x) * kRescoreWarps + warp) * kWarp; b0 < end;
       b0 += static_cast<int64_t>(gridDim.x) * kRescoreWarps * kWarp) {
    const int cnt = static_cast<int>(end - b0 < kWarp ? end - b0 : kWarp);
    int32_t my = lane < cnt ? __ldg(ids + b0 + lane) : 0;
    const bool valid = lane < cnt && my >= 0 && my < n;
    if (lane < cnt && !valid) bad = true;
    if (!valid) my = 0;
    for (int j = 0; j < cnt; ++j) {
      const int32_t idj = __shfl_sync(kFullMask, my, j);
      const float* src = decoded + static_cast<size_t>(idj) * dim;
      for (int t = lane; t < n4; t += kWarp) cp_async16(tile + j * rs + 4 * t, src + 4 * t);
    }
    cp_async_wait_all();
    __syncwarp();
    if (valid) {
      const float4* x4 = reinterpret_cast<const float4*>(tile + lane * rs);
      const float4* q4 = reinterpret_cast<const float4*>(qs);
      float acc = 0.0f;
      for (int t = 0; t < n4; ++t) {
        const float4 x = x4[t];
        const float4 q = q4[t];
        float dl = fsub(q.x, x.x); acc = fadd(acc, fmul(dl, dl));
        dl = fsub(q.y, x.y); acc = fadd(acc, fmul(dl, dl));
        dl = fsub(q.z, x.z); acc = fadd(acc, fmul(dl, dl));
        dl = fsub(q.w, x.w); acc = fadd(acc, fmul(dl, dl));
      }
      if (!isfinite(acc)) bad = true;
      out[b0 + lane] = acc;
    }
    __syncwarp();
  }
  if (bad) status[qi] = kStatusNumeric;
}

// Query codes as retrieval_quantize_query_u8/_u4 produce them
// (l1_int8_core.c:13-63): roundf((q - zero) * (1 / scale)), clamped.
__device__ __forceinline__ void quantize_query(const SqIndexView& ix, const float* q, uint8_t* qc) {
  const float inv = __frcp_rn(ix.l1_scale);
  const int levels = ix.l1_bits == 4 ? 15 : 255;
  for (int d = threadIdx.x; d < ix.dim; d += blockDim.x) {
    int c = static_cast<int>(roundf(fmul(fsub(q[d], ix.l1_zero), inv)));
    qc[d] = static_cast<uint8_t>(c < 0 ? 0 : (c > levels ? levels : c));
  }
}

__global__ void sq_coarse_kernel(SqIndexView ix, const float* __restrict__ queries, int nq,
                                 const int32_t* __restrict__ ids, const int64_t* __restrict__ offsets,
                                 float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(16) uint8_t qc[];
  const int qi = blockIdx.y;
  quantize_query(ix, queries + static_cast<size_t>(qi) * ix.dim, qc);
  __syncthreads();
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  const float scale_sq = fmul(ix.l1_scale, ix.l1_scale);
  bool bad = false;
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = __ldg(ids + i);
    if (id < 0 || id >= ix.n) { bad = true; continue; }
    const uint8_t* x = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
    long long acc = 0;
    if (ix.l1_bits == 8 && (ix.dim & 15) == 0) {
      int iacc = 0;
      for (int d = 0; d < ix.dim; d += 16) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(x + d));
        const uint4 w = *reinterpret_cast<const uint4*>(qc + d);
        iacc += __dp4a(w.x, w.x, 0u) - 2 * static_cast<int>(__dp4a(w.x, v.x, 0u)) + __dp4a(v.x, v.x, 0u);
        iacc += __dp4a(w.y, w.y, 0u) - 2 * static_cast<int>(__dp4a(w.y, v.y, 0u)) + __dp4a(v.y, v.y, 0u);
        iacc += __dp4a(w.z, w.z, 0u) - 2 * static_cast<int>(__dp4a(w.z, v.z, 0u)) + __dp4a(v.z, v.z, 0u);
        iacc += __dp4a(w.w, w.w, 0u) - 2 * static_cast<int>(__dp4a(w.w, v.w, 0u)) + __dp4a(v.w, v.w, 0u);
        if ((d & 1023) == 1008) { acc += iacc; iacc = 0; }
      }
      acc += iacc;
    } else if (ix.l1_bits == 8) {
      for (int d = 0; d < ix.dim; ++d) {
        const int df = static_cast<int>(qc[d]) - static_cast<int>(__ldg(x + d));
        acc += df * df;
      }
    } else {
      for (int d = 0; d < ix.dim; ++d) {
        const int df = static_cast<int>(qc[d] & 15) - nibble(x, d);
        acc += df * df;
      }
    }
    out[i] = fmul(__ll2float_rn(acc), scale_sq);
  }
  if (bad) status[qi] = kStatusBadParam;
}

// The lane side of the split distance (sqmd_dsp_distance_fn with the
// ALIGNED_U8 query contract, retrieval_async_dsp_search.c:993-1016): the
// u8-vs-4-bit L1 distance of each id against the host's aligned query.
__global__ void sq_aligned_coarse_kernel(SqIndexView ix, const uint8_t* __restrict__ queries_u8, int nq,
                                         const int32_t* __restrict__ ids, const int64_t* __restrict__ offsets,
                                         float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(16) uint8_t qu[];
  const int qi = blockIdx.y;
  for (int d = threadIdx.x; d < ix.dim; d += blockDim.x) qu[d] = queries_u8[static_cast<size_t>(qi) * ix.dim + d];
  __syncthreads();
  const double step = split_step(ix.l1_scale);
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  bool bad = false;
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = __ldg(ids + i);
    if (id < 0 || id >= ix.n) { bad = true; continue; }
    out[i] = split_coarse(ix, qu, id, step);
  }
  if (bad) status[qi] = kStatusBadParam;
}

// retrieval_demo_exact_distance_residual_scalar (support.c:1397) of one
// vector: x = (l1*s + z) + (r*rs + rz) per dimension, sequential FP32 sum.
__device__ __forceinline__ float sq_exact_one(const SqIndexView& ix, const float* q, int32_t id) {
  const uint8_t* l1 = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  const uint8_t* res = ix.residual ? ix.residual + static_cast<size_t>(id) * ix.rcb : nullptr;
  float rs = 0.0f, rz = 0.0f, dist = 0.0f;
  if (res) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    rs = qp.x;
    rz = qp.y;
  }
  for (int d = 0; d < ix.dim; ++d) {
    const uint32_t c = ix.l1_bits == 4 ? static_cast<uint32_t>(nibble(l1, d)) : __ldg(l1 + d);
    float value = fadd(fmul(u8f(c), ix.l1_scale), ix.l1_zero);
    if (res) {
      const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, d)) : __ldg(res + d);
      value = fadd(value, fadd(fmul(u8f(r), rs), rz));
    }
    const float diff = fsub(q[d], value);
    dist = fadd(dist, fmul(diff, diff));
  }
  return dist;
}

__global__ void sq_exact_kernel(SqIndexView ix, const float* __restrict__ queries, int nq,
                                const int32_t* __restrict__ ids, const int64_t* __restrict__ offsets,
                                float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(16) float qv[];
  const int qi = blockIdx.y;
  for (int d = threadIdx.x; d < ix.dim; d += blockDim.x) qv[d] = queries[static_cast<size_t>(qi) * ix.dim + d];
  __syncthreads();
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  bool bad = false;
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = __ldg(ids + i);
    if (id < 0 || id >= ix.n) { bad = true; continue; }
    const uint8_t* l1 = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
    const uint8_t* res = ix.residual ? ix.residual + static_cast<size_t>(id) * ix.rcb : nullptr;
    float rs = 0.0f, rz = 0.0f, dist = 0.0f;
    if (res) {
      const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
      rs = qp.x;
      rz = qp.y;
    }
    if (res && ix.l1_bits == 8 && ix.residual_bits == 8 && (ix.dim & 15) == 0) {
      // 8-bit codes and residuals: both rows in 16-byte loads, same order
      for (int d0 = 0; d0 < ix.dim; d0 += 16) {
        const uint4 cv = __ldg(reinterpret_cast<const uint4*>(l1 + d0));
        const uint4 rv = __ldg(reinterpret_cast<const uint4*>(res + d0));
        const uint32_t cw[4] = {cv.x, cv.y, cv.z, cv.w}, rw[4] = {rv.x, rv.y, rv.z, rv.w};
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const uint32_t c = (cw[k >> 2] >> (8 * (k & 3))) & 255u;
          const uint32_t r = (rw[k >> 2] >> (8 * (k & 3))) & 255u;
          const float value = fadd(fadd(fmul(u8f(c), ix.l1_scale), ix.l1_zero), fadd(fmul(u8f(r), rs), rz));
          const float diff = fsub(qv[d0 + k], value);
          dist = fadd(dist, fmul(diff, diff));
        }
      }
      out[i] = dist;
      continue;
    }
    for (int d = 0; d < ix.dim; ++d) {
      const uint32_t c = ix.l1_bits == 4 ? static_cast<uint32_t>(nibble(l1, d)) : __ldg(l1 + d);
      float value = fadd(fmul(u8f(c), ix.l1_scale), ix.l1_zero);
      if (res) {
        const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, d)) : __ldg(res + d);
        value = fadd(value, fadd(fmul(u8f(r), rs), rz));
      }
      const float diff = fsub(qv[d], value);
      dist = fadd(dist, fmul(diff, diff));
    }
    out[i] = dist;
  }
  if (bad) status[qi] = kStatusBadParam;
}

// Decode of one vector for the final refine: PQ  ((c + code*s) + z), SQ
// (l1*ls + lz) + (r*rs + rz), each product and sum rounded to float
// (pq_residual_decode_value :946, retrieval_final_refine_decode_sq :55).
__device__ __forceinline__ bool refine_value(int kind, const PqIndexView& pq, const SqIndexView& sq,
                                             int32_t id, int d, const uint8_t* a, const uint8_t* b,
                                             float2 qp, float* out) {
  float x;
  if (kind == 1) {
    const int m = d / pq.subdim, j = d - m * pq.subdim;
    const int c = pq.ks == 16 ? nibble(a, m) : __ldg(a + m);
    const uint32_t r = pq.residual_bits == 4 ? static_cast<uint32_t>(nibble(b, d)) : __ldg(b + d);
    x = fadd(fadd(__ldg(pq.codebook + (static_cast<size_t>(m) * pq.ks + c) * pq.subdim + j),
                  fmul(u8f(r), qp.x)), qp.y);
  } else {
    const uint32_t c = sq.l1_bits == 4 ? static_cast<uint32_t>(nibble(a, d)) : __ldg(a + d);
    const uint32_t r = sq.residual_bits == 4 ? static_cast<uint32_t>(nibble(b, d)) : __ldg(b + d);
    x = fadd(fadd(fmul(u8f(c), sq.l1_scale), sq.l1_zero), fadd(fmul(u8f(r), qp.x), qp.y));
  }
  *out = x;
  return isfinite(x);
}

// One warp per query: FP64 distances of the candidates on their decoded
// vectors, sorted by (distance, id), top k kept.
__global__ void refine_kernel(int kind, bool error4, PqIndexView pq, SqIndexView sq,
                              const float* __restrict__ decoded, const float* __restrict__ queries,
                              int nq, const int32_t* __restrict__ cand_ids, int cand_stride,
                              const int32_t* __restrict__ cand_counts, int top_k, int capacity,
                              int32_t* out_ids, float* out_dists, int32_t* out_counts, int32_t* status) {
  // mode ERROR4: the index's third-level term on top of every decode
  const Error4View& e4 = kind == 1 ? pq.e4 : sq.e4;
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (qi >= nq) return;
  const int dim = kind == 1 ? pq.dim : sq.dim;
  const int n = kind == 1 ? pq.n : sq.n;
  double* sd = reinterpret_cast<double*>(smem) + static_cast<size_t>(warp) * capacity;
  int32_t* si = reinterpret_cast<int32_t*>(reinterpret_cast<double*>(smem) + static_cast<size_t>(blockDim.x >> 5) * capacity) +
                static_cast<size_t>(warp) * capacity;
  const float* q = queries + static_cast<size_t>(qi) * dim;
  const int count = cand_counts[qi];
  int np2 = 1;
  while (np2 < count) np2 <<= 1;
  bool bad = count < 0 || count > capacity;
  for (int d = lane; d < dim; d += kWarp) bad |= !isfinite(q[d]);
  if (!__any_sync(kFullMask, bad) && kind == 1 && decoded) {
    // the decode read from the decoded rows (NaN rows where the qparams are
    // rejected), 32 candidates at a time staged in shared memory
    const int rs = dim + 4;
    float* tile = reinterpret_cast<float*>(si + static_cast<size_t>((blockDim.x >> 5) - warp) * capacity) +
                  static_cast<size_t>(warp) * kWarp * rs;
    for (int i0 = 0; i0 < np2; i0 += kWarp) {
      const int i = i0 + lane;
      const int cnt = max(0, min(kWarp, count - i0));
      int32_t id = i < count ? cand_ids[static_cast<size_t>(qi) * cand_stride + i] : 0;
      const bool valid = i < count && id >= 0 && id < n;
      if (i < count && !valid) bad = true;
      if (!valid) id = 0;
      for (int j = 0; j < cnt; ++j) {
        const int32_t idj = __shfl_sync(kFullMask, id, j);
        const float* src = decoded + static_cast<size_t>(idj) * dim;
        for (int t = lane; t < dim / 4; t += kWarp) cp_async_chunk<16>(tile + j * rs + 4 * t, src + 4 * t);
      }
      stage_wait();
      __syncwarp();
      if (i < count) {
        double dist = 0.0;
        const float4* x4 = reinterpret_cast<const float4*>(tile + lane * rs);
        const uint8_t* e4c = error4 ? error4_row(e4, id) : nullptr;
        const float2 e4q = e4c ? __ldg(reinterpret_cast<const float2*>(e4.qparams) + id) : make_float2(0.f, 0.f);
        for (int t = 0; t < dim / 4; ++t) {
          const float4 x = x4[t];
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
      } else if (i < np2) {
        sd[i] = __longlong_as_double(0x7ff0000000000000ll);
        si[i] = 0x7fffffff;
      }
      __syncwarp();
    }
  } else if (!__any_sync(kFullMask, bad)) {
    for (int i = lane; i < np2; i += kWarp) {
      if (i < count) {
        const int32_t id = cand_ids[static_cast<size_t>(qi) * cand_stride + i];
        if (id < 0 || id >= n) { bad = true; continue; }
        const uint8_t* a;
        const uint8_t* b;
        float2 qp;
        if (kind == 1) {
          a = pq.codes + static_cast<size_t>(id) * pq.code_bytes;
          b = residual_row(pq, id);
          qp = __ldg(reinterpret_cast<const float2*>(pq.qparams) + id);
          if (!isfinite(qp.x) || !(qp.x > 0.0f) || !isfinite(qp.y)) bad = true;
        } else {
          a = sq.l1 + static_cast<size_t>(id) * sq.l1_code_bytes;
          b = sq.residual + static_cast<size_t>(id) * sq.rcb;
          qp = __ldg(reinterpret_cast<const float2*>(sq.qparams) + id);
          if (!isfinite(sq.l1_scale) || !(sq.l1_scale > 0.0f) || !isfinite(sq.l1_zero) ||
              !isfinite(qp.x) || qp.x < 0.0f || !isfinite(qp.y)) bad = true;
        }
        double dist = 0.0;
        const uint8_t* e4c = error4 ? error4_row(e4, id) : nullptr;
        const float2 e4q = e4c ? __ldg(reinterpret_cast<const float2*>(e4.qparams) + id) : make_float2(0.f, 0.f);
        for (int d = 0; d < dim; ++d) {
          float x;
          if (!refine_value(kind, pq, sq, id, d, a, b, qp, &x)) bad = true;
          if (e4c) {
            x = error4_add(x, e4c, e4q, d);
            if (!isfinite(x)) bad = true;
          }
          const double delta = __dsub_rn(static_cast<double>(q[d]), static_cast<double>(x));
          dist = __dadd_rn(dist, __dmul_rn(delta, delta));
        }
        if (!isfinite(dist) || dist >= 3.4028234663852886e38) bad = true;
        sd[i] = dist;
        si[i] = id;
      } else {
        sd[i] = __longlong_as_double(0x7ff0000000000000ll);
        si[i] = 0x7fffffff;
      }
    }
  }
  if (__any_sync(kFullMask, bad)) {
    if (lane == 0) status[qi] = kStatusNumeric;
    return;
  }
  __syncwarp();
  // duplicate ids are rejected by the reference (refine_impl :269)
  for (int kk = 2; kk <= np2; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < np2; i += kWarp) {
        const int p = i ^ j;
        if (p > i) {
          const bool up = (i & kk) == 0;
          const double x = sd[i], y = sd[p];
          const int32_t ix = si[i], iy = si[p];
          const bool gt = (x > y) || (x == y && ix > iy);
          if (up == gt) { sd[i] = y; sd[p] = x; si[i] = iy; si[p] = ix; }
        }
      }
      __syncwarp();
    }
  }
  bool dup = false;
  for (int i = lane + 1; i < count; i += kWarp) dup |= (si[i] == si[i - 1] && sd[i] == sd[i - 1]);
  if (__any_sync(kFullMask, dup)) {
    if (lane == 0) status[qi] = kStatusBadParam;
    return;
  }
  const int outn = count < top_k ? count : top_k;
  for (int i = lane; i < outn; i += kWarp) {
    out_ids[static_cast<size_t>(qi) * top_k + i] = si[i];
    out_dists[static_cast<size_t>(qi) * top_k + i] = static_cast<float>(sd[i]);
  }
  if (lane == 0) out_counts[qi] = outn;
}

// sq_coarse_kernel / sq_exact_kernel over staged rows (8-bit codes, and for
// the exact distance 8-bit residuals; dim % 16 == 0).
template <bool EXACT>
__global__ void __launch_bounds__(kStageWarps * 32) sq_staged_kernel(SqIndexView ix, const float* __restrict__ queries,
                                                                     int nq, const int32_t* __restrict__ ids,
                                                                     const int64_t* __restrict__ offsets,
                                                                     float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(16) uint8_t smb[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int dim = ix.dim;
  const int RS = stage_stride(dim);
  const int warp_bytes = 128 + 32 * RS + (EXACT ? 32 * RS + 32 * 8 : 0);
  float* qv = reinterpret_cast<float*>(smb);                       // exact: the query
  uint8_t* qc = smb + dim * 4;                                     // coarse: its codes
  uint8_t* wb = smb + dim * 5 + 16 - ((dim * 5) & 15) + warp * warp_bytes;
  int32_t* sid = reinterpret_cast<int32_t*>(wb);
  uint8_t* sl1 = wb + 128;
  uint8_t* sres = sl1 + 32 * RS;
  float2* sqp = reinterpret_cast<float2*>(sres + 32 * RS);
  const int qi = blockIdx.y;
  if (EXACT) {
    for (int d = threadIdx.x; d < dim; d += blockDim.x) qv[d] = queries[static_cast<size_t>(qi) * dim + d];
  } else {
    quantize_query(ix, queries + static_cast<size_t>(qi) * dim, qc);
  }
  __syncthreads();
  const int64_t begin = offsets[qi], end = offsets[qi + 1];
  const float scale_sq = fmul(ix.l1_scale, ix.l1_scale);
  bool bad = false;
  for (int64_t b0 = begin + (static_cast<int64_t>(blockIdx.x) * kStageWarps + warp) * kWarp; b0 < end;
       b0 += static_cast<int64_t>(gridDim.x) * kStageWarps * kWarp) {
    const int cnt = static_cast<int>(end - b0 < kWarp ? end - b0 : kWarp);
    const int32_t my = lane < cnt ? __ldg(ids + b0 + lane) : 0;
    const bool valid = lane < cnt && my >= 0 && my < ix.n;
    if (lane < cnt && !valid) bad = true;
    sid[lane] = valid ? my : 0;
    __syncwarp();
    stage_rows<16>(sl1, RS, dim, cnt, [&](int r) { return ix.l1 + static_cast<size_t>(sid[r]) * dim; }, lane);
    if (EXACT) {
      stage_rows<16>(sres, RS, dim, cnt, [&](int r) { return ix.residual + static_cast<size_t>(sid[r]) * dim; }, lane);
      stage_rows<8>(reinterpret_cast<uint8_t*>(sqp), 8, 8, cnt,
                    [&](int r) { return reinterpret_cast<const uint8_t*>(ix.qparams + 2 * static_cast<size_t>(sid[r])); },
                    lane);
    }
    stage_wait();
    __syncwarp();
    if (valid) {
      const uint4* x = reinterpret_cast<const uint4*>(sl1 + lane * RS);
      if (!EXACT) {
        long long acc = 0;
        int iacc = 0;
        for (int t = 0; t < dim / 16; ++t) {
          const uint4 v = x[t];
          const uint4 w = *reinterpret_cast<const uint4*>(qc + 16 * t);
          iacc += __dp4a(w.x, w.x, 0u) - 2 * static_cast<int>(__dp4a(w.x, v.x, 0u)) + __dp4a(v.x, v.x, 0u);
          iacc += __dp4a(w.y, w.y, 0u) - 2 * static_cast<int>(__dp4a(w.y, v.y, 0u)) + __dp4a(v.y, v.y, 0u);
          iacc += __dp4a(w.z, w.z, 0u) - 2 * static_cast<int>(__dp4a(w.z, v.z, 0u)) + __dp4a(v.z, v.z, 0u);
          iacc += __dp4a(w.w, w.w, 0u) - 2 * static_cast<int>(__dp4a(w.w, v.w, 0u)) + __dp4a(v.w, v.w, 0u);
          if ((t & 63) == 63) { acc += iacc; iacc = 0; }
        }
        acc += iacc;
        out[b0 + lane] = fmul(__ll2float_rn(acc), scale_sq);
      } else {
        const uint4* rr = reinterpret_cast<const uint4*>(sres + lane * RS);
        const float2 qp = sqp[lane];
        float dist = 0.0f;
        for (int t = 0; t < dim / 16; ++t) {
          const uint4 cv = x[t], rv = rr[t];
          const uint32_t cw[4] = {cv.x, cv.y, cv.z, cv.w}, rw[4] = {rv.x, rv.y, rv.z, rv.w};
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const uint32_t c = (cw[k >> 2] >> (8 * (k & 3))) & 255u;
            const uint32_t r = (rw[k >> 2] >> (8 * (k & 3))) & 255u;
            const float value = fadd(fadd(fmul(u8f(c), ix.l1_scale), ix.l1_zero), fadd(fmul(u8f(r), qp.x), qp.y));
            const float diff = fsub(qv[16 * t + k], value);
            dist = fadd(dist, fmul(diff, diff));
          }
        }
        out[b0 + lane] = dist;
      }
    }
    __syncwarp();
  }
  if (bad) status[qi] = kStatusBadParam;
}

size_t sq_staged_smem(int dim, bool exact) {
  const int rs = ((((dim + 15) / 16) | 1) * 16);
  return static_cast<size_t>(dim) * 5 + 16 + static_cast<size_t>(kStageWarps) * (128 + 32 * rs + (exact ? 32 * rs + 256 : 0));
}

// demo_rerank_candidates (retrieval_rpc_demo_support.c:1833-1862), the
// legacy SQ re-rank, one warp per query: a stable insertion sort by id, the
// exact residual distance of every candidate (FLT_MAX for an id outside the
// index), a stable insertion sort by distance, the first top_k.  Both stable
// sorts are bitonic sorts of (key, position) pairs, which order exactly as
// the insertion sorts do while every distance compares; when a distance is
// NaN (the insertion sort then stops at it) lane 0 replays the insertion
// sort itself.  No reorder map: the id is the sort key.
__global__ void rerank_kernel(SqIndexView ix, const float* __restrict__ queries, int nq,
                              const int32_t* __restrict__ cand_ids, int cand_stride,
                              const int32_t* __restrict__ cand_counts, int top_k, int capacity, int32_t* out_ids,
                              float* out_dists, int32_t* out_counts, int32_t* status) {
  extern __shared__ __align__(16) uint8_t rsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qi = blockIdx.x * (blockDim.x >> 5) + warp;
  if (qi >= nq) return;
  uint64_t* key = reinterpret_cast<uint64_t*>(rsm) + static_cast<size_t>(warp) * capacity;
  float* dist = reinterpret_cast<float*>(reinterpret_cast<uint64_t*>(rsm) + static_cast<size_t>(blockDim.x >> 5) * capacity) +
                static_cast<size_t>(warp) * capacity;
  int32_t* ids = reinterpret_cast<int32_t*>(dist + static_cast<size_t>((blockDim.x >> 5) - warp) * capacity) +
                 static_cast<size_t>(warp) * capacity;
  const float* q = queries + static_cast<size_t>(qi) * ix.dim;
  const int count = cand_counts[qi];
  if (count < 0 || count > capacity) {
    if (lane == 0) status[qi] = kStatusBadParam;
    return;
  }
  int np2 = 1;
  while (np2 < count) np2 <<= 1;
  auto bitonic = [&]() {
    for (int kk = 2; kk <= np2; kk <<= 1)
      for (int j = kk >> 1; j > 0; j >>= 1) {
        for (int i = lane; i < np2; i += kWarp) {
          const int p = i ^ j;
          if (p > i) {
            const bool up = (i & kk) == 0;
            const uint64_t a = key[i], b = key[p];
            if (up == (a > b)) { key[i] = b; key[p] = a; }
          }
        }
        __syncwarp();
      }
  };
  // stable by id: (signed id, position)
  for (int i = lane; i < np2; i += kWarp) {
    if (i < count) {
      const uint32_t id = static_cast<uint32_t>(cand_ids[static_cast<size_t>(qi) * cand_stride + i]) ^ 0x80000000u;
      key[i] = (static_cast<uint64_t>(id) << 32) | static_cast<uint32_t>(i);
    } else {
      key[i] = ~0ull;
    }
  }
  __syncwarp();
  bitonic();
  bool nan = false;
  for (int i = lane; i < count; i += kWarp) {
    const int32_t id = static_cast<int32_t>(static_cast<uint32_t>(key[i] >> 32) ^ 0x80000000u);
    const float d = (id < 0 || id >= ix.n) ? 3.40282346638528859812e+38f : sq_exact_one(ix, q, id);
    ids[i] = id;
    dist[i] = d;
    nan |= isnan(d);
  }
  __syncwarp();
  if (!__any_sync(kFullMask, nan)) {
    // stable by distance: (distance bits, rank after the id sort); the
    // distances are sums of squares (>= +0) or FLT_MAX / inf
    for (int i = lane; i < np2; i += kWarp)
      key[i] = i < count ? (static_cast<uint64_t>(__float_as_uint(dist[i])) << 32) | static_cast<uint32_t>(i) : ~0ull;
    __syncwarp();
    bitonic();
    const int outn = count < top_k ? count : top_k;
    for (int i = lane; i < outn; i += kWarp) {
      const int r = static_cast<int>(key[i] & 0xffffffffu);
      out_ids[static_cast<size_t>(qi) * top_k + i] = ids[r];
      out_dists[static_cast<size_t>(qi) * top_k + i] = dist[r];
    }
    if (lane == 0) out_counts[qi] = outn;
    return;
  }
  if (lane == 0) {
    for (int j = 1; j < count; ++j) {
      const int32_t tid = ids[j];
      const float tdt = dist[j];
      int k = j - 1;
      while (k >= 0 && dist[k] > tdt) {
        ids[k + 1] = ids[k];
        dist[k + 1] = dist[k];
        --k;
      }
      ids[k + 1] = tid;
      dist[k + 1] = tdt;
    }
    const int outn = count < top_k ? count : top_k;
    for (int i = 0; i < outn; ++i) {
      out_ids[static_cast<size_t>(qi) * top_k + i] = ids[i];
      out_dists[static_cast<size_t>(qi) * top_k + i] = dist[i];
    }
    out_counts[qi] = outn;
  }
}

// ---------------------------------------------------------------------------

void launch_pq_lut(const PqIndexView& ix, const float* queries, int nq, float* luts,
                   int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  pq_lut_kernel<<<nq, 256, 0, s>>>(ix, queries, nq, luts, status);
}

void launch_pq_adc(const PqIndexView& ix, const float* luts, int nq, const int32_t* ids,
                   const int64_t* offsets, float* out, int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  const size_t smem = static_cast<size_t>(ix.m) * ix.ks * sizeof(float);
  if (smem > 48 * 1024) cudaFuncSetAttribute(pq_adc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  dim3 grid(8, nq);
  pq_adc_kernel<<<grid, 256, smem, s>>>(ix, luts, nq, ids, offsets, out, status);
}

void launch_pq_residual(const PqIndexView& ix, const float* queries, int nq, const int32_t* ids,
                        const int64_t* offsets, float* out, int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  dim3 grid(8, nq);
  const size_t smem = ix.dim * sizeof(float);
  if (ix.ks == 256 && ix.code_bytes == ix.m && (ix.residual_bits == 8 || ix.residual_bits == 4)) {
    const bool r8 = ix.residual_bits == 8;
#define ROVER_RES_SHAPE(MM, SS)                                                                               \
  if (ix.m == MM && ix.subdim == SS) {                                                                        \
    if (r8) pq_residual_kernel<MM, SS, 8><<<grid, 128, smem, s>>>(ix, queries, nq, ids, offsets, out, status); \
    else pq_residual_kernel<MM, SS, 4><<<grid, 128, smem, s>>>(ix, queries, nq, ids, offsets, out, status);    \
    return;                                                                                                   \
  }
    ROVER_RES_SHAPE(16, 8)
    ROVER_RES_SHAPE(32, 4)
    ROVER_RES_SHAPE(24, 4)
    ROVER_RES_SHAPE(8, 8)
    ROVER_RES_SHAPE(16, 4)
#undef ROVER_RES_SHAPE
  }
  pq_residual_kernel<0, 0, 0><<<grid, 128, smem, s>>>(ix, queries, nq, ids, offsets, out, status);
}

void launch_pq_rescore(int dim, int n, const float* decoded, const float* queries, int nq, const int32_t* ids,
                       const int64_t* offsets, float* out, int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  const size_t smem = (static_cast<size_t>(dim) + static_cast<size_t>(kRescoreWarps) * kWarp * (dim + 4)) * sizeof(float);
  cudaFuncSetAttribute(pq_rescore_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  dim3 grid(8, nq);
  pq_rescore_kernel<<<grid, kRescoreWarps * 32, smem, s>>>(dim, n, decoded, queries, nq, ids, offsets, out, status);
}

void launch_sq_coarse(const SqIndexView& ix, const float* queries, int nq, const int32_t* ids,
                      const int64_t* offsets, float* out, int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  dim3 grid(8, nq);
  if (ix.l1_bits == 8 && (ix.dim & 15) == 0 && sq_staged_smem(ix.dim, false) <= 227 * 1024) {
    const size_t smem = sq_staged_smem(ix.dim, false);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(sq_staged_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    sq_staged_kernel<false><<<grid, kStageWarps * 32, smem, s>>>(ix, queries, nq, ids, offsets, out, status);
    return;
  }
  sq_coarse_kernel<<<grid, 128, (ix.dim + 15) & ~15, s>>>(ix, queries, nq, ids, offsets, out, status);
}

void launch_sq_aligned_coarse(const SqIndexView& ix, const uint8_t* queries_u8, int nq, const int32_t* ids,
                              const int64_t* offsets, float* out, int32_t* status, cudaStream_t s) {
  if (nq <= 0 || ix.l1_bits != 4) return;
  dim3 grid(8, nq);
  sq_aligned_coarse_kernel<<<grid, 128, (ix.dim + 15) & ~15, s>>>(ix, queries_u8, nq, ids, offsets, out, status);
}

void launch_sq_exact(const SqIndexView& ix, const float* queries, int nq, const int32_t* ids,
                     const int64_t* offsets, float* out, int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  dim3 grid(8, nq);
  if (ix.l1_bits == 8 && ix.residual && ix.residual_bits == 8 && ix.rcb == ix.dim && (ix.dim & 15) == 0 &&
      sq_staged_smem(ix.dim, true) <= 227 * 1024) {
    const size_t smem = sq_staged_smem(ix.dim, true);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(sq_staged_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    sq_staged_kernel<true><<<grid, kStageWarps * 32, smem, s>>>(ix, queries, nq, ids, offsets, out, status);
    return;
  }
  sq_exact_kernel<<<grid, 128, ix.dim * sizeof(float), s>>>(ix, queries, nq, ids, offsets, out, status);
}

void launch_rerank(const SqIndexView& ix, const float* queries, int nq, const int32_t* cand_ids, int cand_stride,
                   const int32_t* cand_counts, int top_k, int capacity, int32_t* out_ids, float* out_dists,
                   int32_t* out_counts, int32_t* status, cudaStream_t s) {
  if (nq <= 0) return;
  int cap = 1;
  while (cap < capacity) cap <<= 1;
  const int warps = cap <= 1024 ? 4 : 1;
  const size_t smem = static_cast<size_t>(warps) * cap * 16;
  if (smem > 48 * 1024) cudaFuncSetAttribute(rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  rerank_kernel<<<(nq + warps - 1) / warps, warps * 32, smem, s>>>(ix, queries, nq, cand_ids, cand_stride, cand_counts,
                                                                   top_k, cap, out_ids, out_dists, out_counts, status);
}

void launch_refine(int kind, const PqIndexView& pq, const SqIndexView& sq, const float* decoded, const float* queries,
                   int nq, const int32_t* cand_ids, int cand_stride, const int32_t* cand_counts,
                   int top_k, int capacity, int32_t* out_ids, float* out_dists,
                   int32_t* out_counts, int32_t* status, cudaStream_t s, bool error4) {
  if (nq <= 0) return;
  int cap = 1;
  while (cap < capacity) cap <<= 1;
  const int warps = 4;
  const int dim = kind == 1 ? pq.dim : sq.dim;
  size_t smem = static_cast<size_t>(warps) * cap * 12;
  if (kind == 1 && decoded) smem += static_cast<size_t>(warps) * kWarp * (dim + 4) * sizeof(float);
  if (smem > 227 * 1024 && kind == 1 && decoded) {   // tile too large: decode per element instead
    decoded = nullptr;
    smem = static_cast<size_t>(warps) * cap * 12;
  }
  if (smem > 48 * 1024) cudaFuncSetAttribute(refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  refine_kernel<<<(nq + warps - 1) / warps, warps * 32, smem, s>>>(kind, error4, pq, sq, decoded, queries, nq, cand_ids,
                                                                   cand_stride,
                                                                   cand_counts, top_k, cap, out_ids, out_dists,
                                                                   out_counts, status);
}

}  // namespace rover
