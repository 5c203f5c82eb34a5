// common.cuh -- device-side building blocks shared by the search kernels.
//
// Numerics: every FP32 step that the reference evaluates as a separate
// rounded operation is written with the _rn intrinsics, which the compiler
// never contracts into FMA, so distances are bit-identical to the reference
// host build (which is compiled without FP contraction).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rover {

constexpr int kWarp = 32;
constexpr uint32_t kFullMask = 0xffffffffu;

// Per-query status codes written by the search kernels.
enum QueryStatus : int32_t {
  kStatusOk = 0,
  kStatusBadRow = 1,        // graph row violates the valid-prefix rule
  kStatusNumeric = 2,       // non-finite distance / invalid qparams
  kStatusTableFull = 3,     // visited table exceeded its load limit
  kStatusBadParam = 4,      // request out of range (pool, k, expand, ids)
  kStatusFrontierFull = 5,  // SQ frontier exceeded the reference's bound
  kStatusSeedRank = 6,      // the tensor-core seed ranking of the launch gave up waiting (bounded waits)
};

// The final refine's third-level ERROR4 term (retrieval_final_refine.c:
// 118-166, :221-246): per storage row an int4 code per dimension, packed
// low nibble first into ceil(dim/2) bytes, vpb rows per 4096-byte block, and
// a {scale, zero} pair.  qparams == nullptr when no artifact is loaded.
struct Error4View {
  const float* qparams;     // [n][2]
  const uint8_t* blocks;
  int32_t code_bytes, vpb;
};

struct PqIndexView {
  const int32_t* graph;     // [n][degree]
  int32_t n, degree, dim;
  const uint8_t* codes;     // [n][code_bytes]
  const float* codebook;    // [m][ks][subdim]
  int32_t m, ks, subdim, code_bytes;
  const uint8_t* residual;  // 4096-byte blocks of vpb rows each
  int32_t residual_bits, rcb, vpb;
  const float* qparams;     // [n][2] {scale, zero}
  float codebook_absmax;    // max |codebook entry| (bounds every LUT entry)
  Error4View e4;            // ERROR4 artifact of this index (optional)
};

struct SqIndexView {
  const int32_t* graph;
  int32_t n, degree, dim;
  const uint8_t* l1;        // [n][l1_code_bytes]
  int32_t l1_bits, l1_code_bytes;
  float l1_scale, l1_zero;
  const uint8_t* residual;  // [n][rcb] flat rows (may be null)
  int32_t residual_bits, rcb;
  const float* qparams;     // [n][2]
  Error4View e4;            // ERROR4 artifact of this index (optional)
  const float* split_bias;  // [n] SQ4 split-distance bias (optional)
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

__device__ __forceinline__ int nibble(const uint8_t* p, int i) {
  const int b = p[i >> 1];
  return (i & 1) ? (b >> 4) : (b & 15);
}

// decode_vector's ERROR4 step for dimension d of one row: x + (code * scale
// + zero), each product and sum rounded to float (decode_value, add_f32).
__device__ __forceinline__ float error4_add(float x, const uint8_t* codes, float2 qp, int d);

// Exact small-integer to float: byte b -> float(b) by placing b in the
// mantissa of 2^23 and subtracting 2^23 (exact for b < 2^23).
__device__ __forceinline__ float u8f(uint32_t b) {
  return __fsub_rn(__uint_as_float(0x4B000000u | b), 8388608.0f);
}

__device__ __forceinline__ float error4_add(float x, const uint8_t* codes, float2 qp, int d) {
  return fadd(x, fadd(fmul(u8f(static_cast<uint32_t>(nibble(codes, d))), qp.x), qp.y));
}

// The ERROR4 codes of storage row `row`.
__device__ __forceinline__ const uint8_t* error4_row(const Error4View& e, int32_t row) {
  return e.blocks + static_cast<size_t>(row / e.vpb) * 4096u + static_cast<size_t>(row % e.vpb) * e.code_bytes;
}

// Candidate keys: (distance bits << 32) | id.  Distances are squared norms
// (>= +0), so their IEEE bits order like the values; the 64-bit key then
// orders by (distance, id) exactly as the reference's strict total order
// (retrieval_sqmd_pure_pq.c:97-112).  Bit 31 of the id word marks
// "already expanded" and is masked out of comparisons.
constexpr uint64_t kExpandedBit = 0x80000000ull;
constexpr uint64_t kEmptyKey = ~0ull;

__device__ __forceinline__ uint64_t make_key(float d, int32_t id) {
  return (static_cast<uint64_t>(__float_as_uint(d)) << 32) | static_cast<uint32_t>(id);
}
__device__ __forceinline__ uint64_t key_cmp(uint64_t k) { return k & ~kExpandedBit; }
__device__ __forceinline__ int32_t key_id(uint64_t k) {
  return static_cast<int32_t>(static_cast<uint32_t>(k) & 0x7fffffffu);
}
__device__ __forceinline__ float key_dist(uint64_t k) {
  return __uint_as_float(static_cast<uint32_t>(k >> 32));
}

// ---------------------------------------------------------------------------
// Visited set: open-addressing table of 64-bit entries (generation << 32 | id)
// in global memory, one table per warp slot.  An entry whose generation is
// not the current query's counts as empty, so tables never need clearing
// between queries: a query only ever turns stale entries into current ones,
// which keeps linear probing exact.
struct VisitedTable {
  unsigned long long* slots;
  uint32_t mask;   // capacity - 1 (capacity is a power of two)
  uint32_t gen;    // current query generation (never 0 for a live query)
};

__device__ __forceinline__ uint32_t hash_id(uint32_t id) {
  // murmur3 finalizer
  id ^= id >> 16; id *= 0x85ebca6bu; id ^= id >> 13; id *= 0xc2b2ae35u; id ^= id >> 16;
  return id;
}

// Returns 1 if id was inserted now (first visit), 0 if it was already
// present, -1 if the probe sequence exceeded the table (caller reports it).
__device__ __forceinline__ int visited_insert(const VisitedTable& t, uint32_t id) {
  const unsigned long long want = (static_cast<unsigned long long>(t.gen) << 32) | id;
  uint32_t h = hash_id(id) & t.mask;
  for (uint32_t probe = 0; probe <= t.mask; ++probe) {
    unsigned long long cur = *(volatile unsigned long long*)&t.slots[h];
    while (static_cast<uint32_t>(cur >> 32) != t.gen) {
      const unsigned long long prev = atomicCAS(&t.slots[h], cur, want);
      if (prev == cur) return 1;
      cur = prev;
    }
    if (cur == want) return 0;
    h = (h + 1) & t.mask;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// Warp-wide bitonic sort of up to 32*PER keys held PER per lane (ascending),
// element index e = lane + 32*r for register r.
template <int PER>
__device__ __forceinline__ void warp_bitonic_sort(uint64_t (&v)[PER], int lane) {
  constexpr int N = 32 * PER;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int rj = j / 32;
#pragma unroll
        for (int r = 0; r < PER; ++r) {
          const int partner = r ^ rj;
          if (partner > r) {
            const int e = lane + 32 * r;
            const bool up = (e & k) == 0;
            const uint64_t a = v[r], b = v[partner];
            const bool swap = up ? (key_cmp(a) > key_cmp(b)) : (key_cmp(a) < key_cmp(b));
            if (swap) { v[r] = b; v[partner] = a; }
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < PER; ++r) {
          const int e = lane + 32 * r;
          const uint64_t other = __shfl_xor_sync(kFullMask, v[r], j);
          const bool up = (e & k) == 0;
          const bool lower = (lane & j) == 0;
          const uint64_t a = v[r];
          const bool take_min = (lower == up);
          const bool a_less = key_cmp(a) < key_cmp(other);
          v[r] = take_min ? (a_less ? a : other) : (a_less ? other : a);
        }
      }
    }
  }
}

// Number of keys in sorted smem array a[0..n) that compare below key.
__device__ __forceinline__ int count_less(const uint64_t* a, int n, uint64_t key) {
  const uint64_t k = key_cmp(key);
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (key_cmp(a[mid]) < k) lo = mid + 1; else hi = mid;
  }
  return lo;
}

}  // namespace rover
