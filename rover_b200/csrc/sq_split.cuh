// sq_split.cuh -- the SQ4 split distance (SQMD_SPLIT_DISTANCE on).
//
// The reference splits the SQMD correction in two: the lanes compute an L1
// code distance against a query quantized on the 4-bit L1 grid refined
// 17-fold (retrieval_quantize_query_l1_aligned_u8 and
// retrieval_compute_u8_u4_l1_distance_scalar, retrieval_l1_int8_core.c:
// 65-111, :171-191), and the host adds a per-vector delta bias[id] - 2 q.r
// whose dot product is expanded over integer sums (sqmd_split_residual_
// delta_fn, retrieval_rpc_demo_pipeline.c:935-976, over retrieval_compute_
// u8_u4 / u8_u8_residual_dot_scalar, retrieval_l1_int8_core.c:193-263).
// The bias (sum of 2 a r + r^2 per vector) comes precomputed from the index
// build.  Every double operation below is the reference's, in its order, as
// a separately rounded intrinsic.
#pragma once

#include "common.cuh"

namespace rover {

// (double)l1_scale / 17: the step of the refined grid.
__device__ __forceinline__ double split_step(float l1_scale) {
  return __ddiv_rn(static_cast<double>(l1_scale), 17.0);
}

// One dimension of the aligned u8 query: lround((v - zero) / step) clamped to
// 0..255 (lround rounds half away from zero).  False on a non-finite input.
__device__ __forceinline__ bool split_code(float v, float zero, double step, uint8_t* code) {
  const double raw = __ddiv_rn(__dsub_rn(static_cast<double>(v), static_cast<double>(zero)), step);
  if (!isfinite(v) || !isfinite(raw)) return false;
  int c;
  if (raw <= 0.0) {
    c = 0;                       // rounds to <= 0, clamped
  } else if (raw >= 255.5) {
    c = 255;                     // rounds to >= 256, clamped
  } else {
    const double t = trunc(raw);
    c = static_cast<int>(t) + (__dsub_rn(raw, t) >= 0.5 ? 1 : 0);
  }
  *code = static_cast<uint8_t>(c);
  return true;
}

// The lanes' L1 distance: sum (q - 17 code)^2 as an integer, then
// (float)(acc * step * step) in double.
__device__ __forceinline__ float split_coarse(const SqIndexView& ix, const uint8_t* qu, int32_t id, double step) {
  const uint8_t* x = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  long long acc = 0;
  for (int d = 0; d < ix.dim; ++d) {
    const int diff = static_cast<int>(qu[d]) - 17 * nibble(x, d);
    acc += static_cast<long long>(diff) * diff;
  }
  return __double2float_rn(__dmul_rn(__dmul_rn(__ll2double_rn(acc), step), step));
}

// The host's delta bias[id] - 2 <q, r>; NaN when the row's parameters are
// invalid or the result is not finite.
__device__ __forceinline__ float split_delta(const SqIndexView& ix, const uint8_t* qu, unsigned long long sum_q,
                                             int32_t id, double step) {
  const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
  if (!isfinite(ix.l1_scale) || !isfinite(ix.l1_zero) || !isfinite(qp.x) || !isfinite(qp.y) ||
      !(ix.l1_scale > 0.0f) || qp.x < 0.0f)
    return __int_as_float(0x7fc00000);
  const uint8_t* r = ix.residual + static_cast<size_t>(id) * ix.rcb;
  unsigned long long sqv = 0, sv = 0;
  for (int d = 0; d < ix.dim; ++d) {
    const unsigned v = ix.residual_bits == 4 ? static_cast<unsigned>(nibble(r, d)) : __ldg(r + d);
    sqv += static_cast<unsigned long long>(qu[d]) * v;
    sv += v;
  }
  const double lz = static_cast<double>(ix.l1_zero), rs = static_cast<double>(qp.x), rz = static_cast<double>(qp.y);
  double dot = __dmul_rn(__dmul_rn(step, rs), __ull2double_rn(sqv));
  dot = __dadd_rn(dot, __dmul_rn(__dmul_rn(step, rz), __ull2double_rn(sum_q)));
  dot = __dadd_rn(dot, __dmul_rn(__dmul_rn(lz, rs), __ull2double_rn(sv)));
  dot = __dadd_rn(dot, __dmul_rn(__dmul_rn(static_cast<double>(ix.dim), lz), rz));
  const double delta = __dsub_rn(static_cast<double>(__ldg(ix.split_bias + id)), __dmul_rn(2.0, dot));
  return isfinite(delta) ? __double2float_rn(delta) : __int_as_float(0x7fc00000);
}

// coarse + delta with the reference's clamp of tiny negative sums to zero.
__device__ __forceinline__ float split_sum(float coarse, float delta) {
  float d = fadd(coarse, delta);
  if (d < 0.0f && d > -1.0e-4f) d = 0.0f;
  return d;
}

// sqmd_split_distance_for_id (retrieval_rpc_demo_pipeline.c:978-995), the
// seeds' distance: FLT_MAX when either part is not finite.
__device__ __forceinline__ float split_seed_distance(const SqIndexView& ix, const uint8_t* qu,
                                                     unsigned long long sum_q, int32_t id, double step) {
  const float c = split_coarse(ix, qu, id, step);
  const float dl = split_delta(ix, qu, sum_q, id, step);
  if (!isfinite(c) || !isfinite(dl)) return 3.402823466e+38f;
  return split_sum(c, dl);
}

}  // namespace rover
