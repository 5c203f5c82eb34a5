// sq_search.cu -- SQ beam search with the reference's exact heap semantics.
//
// Two reference loops are served:
//  * kSqModeDsp: calculator_retrieval_search, the legacy full device search
//    (src/dsp_demo/retrieval_async_dsp_search.c:368-509): LCG entries
//    (dsp_search_select_entry_id :219), neighbours outside [0, n) skipped one
//    by one, coarse SQ distances only.
//  * kSqModeSqmd: the CLI's SQMD loop (retrieval_sqmd_common.c
//    sqmd_cpu_state_run_fake_dsp :2052 with dispatch :283 and apply :638),
//    seeds from retrieval_sqmd_make_seed_ids (retrieval_sqmd_seed.c:15), and
//    the exact residual distance (retrieval_rpc_demo_support.c:1397) replacing
//    the coarse one when correction is on.
//  * kSqModeDb: one query of calculator_retrieval_search_db, the DB-pair
//    search (retrieval_async_dsp_search.c:1205-1581): the device search of
//    kSqModeDsp (entries, pool clamp, neighbour filtering), except that every
//    expansion candidate enters the pool with the distance the host's
//    correction thread returns for it (retrieval_rpc_demo_pipeline.c:454-495:
//    the exact residual distance with correction on, the coarse one with it
//    off) and that the frontier grows as needed (db_search_reserve_frontier).
//
// SQ pool and frontier heaps order by distance only and break ties by heap
// position (strict '<' replacement, sqmd_common.c:51-80), so results depend
// on the insertion order.  The kernel therefore keeps the reference's heaps
// verbatim: one warp per query computes distances in parallel, lane 0 applies
// the heap operations in the reference's order.

#include "common.cuh"
#include "kernels.h"
#include "sq_split.cuh"

namespace rover {

struct HeapEntry { int32_t id; float dist; };

// A heap whose first `split` entries sit in this warp's shared memory and
// whose deeper entries sit at the same indices of its global scratch: the
// levels every push and pop touches stay on chip, and a large frontier (the
// SQMD bound is entry points + pool x expand) still fits.
struct SplitHeap {
  HeapEntry* sm;
  HeapEntry* gl;
  int split;
  __device__ __forceinline__ HeapEntry& operator[](int i) const { return i < split ? sm[i] : gl[i]; }
};

template <class H>
__device__ __forceinline__ void pool_sift_up(H p, int i) {
  HeapEntry t = p[i];
  while (i > 0) {
    const int parent = (i - 1) / 2;
    if (t.dist <= p[parent].dist) break;
    p[i] = p[parent];
    i = parent;
  }
  p[i] = t;
}

template <class H>
__device__ __forceinline__ void pool_sift_down(H p, int size, int i) {
  HeapEntry t = p[i];
  for (;;) {
    int child = 2 * i + 1;
    if (child >= size) break;
    if (child + 1 < size && p[child + 1].dist > p[child].dist) ++child;
    if (t.dist >= p[child].dist) break;
    p[i] = p[child];
    i = child;
  }
  p[i] = t;
}

template <class H>
__device__ __forceinline__ bool pool_insert(H p, int* size, int cap, int32_t id, float d) {
  if (*size < cap) {
    p[*size] = HeapEntry{id, d};
    pool_sift_up(p, *size);
    ++*size;
    return true;
  }
  if (d < p[0].dist) {
    p[0] = HeapEntry{id, d};
    pool_sift_down(p, *size, 0);
    return true;
  }
  return false;
}

template <class H>
__device__ __forceinline__ void front_sift_up(H f, int i) {
  HeapEntry t = f[i];
  while (i > 0) {
    const int parent = (i - 1) / 2;
    if (t.dist >= f[parent].dist) break;
    f[i] = f[parent];
    i = parent;
  }
  f[i] = t;
}

template <class H>
__device__ __forceinline__ void front_sift_down(H f, int size, int i) {
  HeapEntry t = f[i];
  for (;;) {
    int child = 2 * i + 1;
    if (child >= size) break;
    if (child + 1 < size && f[child + 1].dist < f[child].dist) ++child;
    if (t.dist <= f[child].dist) break;
    f[i] = f[child];
    i = child;
  }
  f[i] = t;
}

template <class H>
__device__ __forceinline__ int32_t front_pop(H f, int* size) {
  const int32_t top = f[0].id;
  --*size;
  if (*size > 0) {
    f[0] = f[*size];
    front_sift_down(f, *size, 0);
  }
  return top;
}

// retrieval_compute_int8_native_distance_u8_scalar / int4_packed (l1_int8_core.c:119-169):
// exact integer sum of squared code differences, then (float)acc * scale^2.
__device__ __forceinline__ float sq_coarse(const SqIndexView& ix, const uint8_t* qc, int32_t id) {
  const uint8_t* x = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  long long acc = 0;
  if (ix.l1_bits == 8) {
    int d = 0;
    if ((ix.dim & 3) == 0) {
      const uint32_t* xw = reinterpret_cast<const uint32_t*>(x);
      const uint32_t* qw = reinterpret_cast<const uint32_t*>(qc);
      int iacc = 0;
      for (; d < ix.dim; d += 4) {
        const uint32_t a = qw[d >> 2];
        const uint32_t b = __ldg(xw + (d >> 2));
        // sum (a_i - b_i)^2 = sum a^2 - 2 sum ab + sum b^2, exact in int32 per word
        iacc += __dp4a(a, a, 0u) - 2 * static_cast<int>(__dp4a(a, b, 0u)) + __dp4a(b, b, 0u);
        if ((d & 1023) == 1020) { acc += iacc; iacc = 0; }
      }
      acc += iacc;
    } else {
      for (; d < ix.dim; ++d) {
        const int df = static_cast<int>(qc[d]) - static_cast<int>(__ldg(x + d));
        acc += df * df;
      }
    }
  } else {
    for (int d = 0; d < ix.dim; ++d) {
      const int df = static_cast<int>(qc[d] & 15) - nibble(x, d);
      acc += df * df;
    }
  }
  const float scale_sq = fmul(ix.l1_scale, ix.l1_scale);
  return fmul(__ll2float_rn(acc), scale_sq);
}

// retrieval_demo_exact_distance_residual_scalar (support.c:1397-1443)
__device__ __forceinline__ float sq_exact(const SqIndexView& ix, const float* q, int32_t id) {
  const uint8_t* l1 = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  const uint8_t* res = ix.residual ? ix.residual + static_cast<size_t>(id) * ix.rcb : nullptr;
  float rs = 0.0f, rz = 0.0f, dist = 0.0f;
  if (res) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    rs = qp.x;
    rz = qp.y;
  }
  for (int i = 0; i < ix.dim; ++i) {
    const uint32_t c = ix.l1_bits == 4 ? static_cast<uint32_t>(nibble(l1, i)) : __ldg(l1 + i);
    float value = fadd(fmul(u8f(c), ix.l1_scale), ix.l1_zero);
    if (res) {
      const uint32_t r = ix.residual_bits == 4 ? static_cast<uint32_t>(nibble(res, i)) : __ldg(res + i);
      value = fadd(value, fadd(fmul(u8f(r), rs), rz));
    }
    const float diff = fsub(q[i], value);
    dist = fadd(dist, fmul(diff, diff));
  }
  return dist;
}

// Code of dimension j (0..15) of a 16-dimension group held in v: 4-bit codes
// (64 bits, low nibble first) or 8-bit codes (128 bits).
__device__ __forceinline__ uint32_t group_code(const uint4& v, bool four, int j) {
  if (four) {
    const uint32_t w = j < 8 ? v.x : v.y;
    return (w >> ((j & 7) * 4)) & 15u;
  }
  const uint32_t w = j < 4 ? v.x : j < 8 ? v.y : j < 12 ? v.z : v.w;
  return (w >> ((j & 3) * 8)) & 255u;
}

__device__ __forceinline__ uint4 group_load(const uint8_t* row, bool four, int g) {
  if (four) {
    const uint2 t = __ldg(reinterpret_cast<const uint2*>(row + g / 2));
    return make_uint4(t.x, t.y, 0u, 0u);
  }
  return __ldg(reinterpret_cast<const uint4*>(row + g));
}

// sq_exact over 16-dimension groups read with 64/128-bit loads (rows whose
// code and residual strides keep those loads aligned, dim % 16 == 0): the
// same per-dimension arithmetic, in dimension order.
__device__ __forceinline__ float sq_exact_vec(const SqIndexView& ix, const float* q, int32_t id) {
  const uint8_t* l1 = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  const uint8_t* res = ix.residual ? ix.residual + static_cast<size_t>(id) * ix.rcb : nullptr;
  const bool c4 = ix.l1_bits == 4, r4 = ix.residual_bits == 4;
  float rs = 0.0f, rz = 0.0f, dist = 0.0f;
  if (res) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    rs = qp.x;
    rz = qp.y;
  }
  for (int g = 0; g < ix.dim; g += 16) {
    const uint4 cv = group_load(l1, c4, g);
    const uint4 rv = res ? group_load(res, r4, g) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      float value = fadd(fmul(u8f(group_code(cv, c4, j)), ix.l1_scale), ix.l1_zero);
      if (res) value = fadd(value, fadd(fmul(u8f(group_code(rv, r4, j)), rs), rz));
      const float diff = fsub(q[g + j], value);
      dist = fadd(dist, fmul(diff, diff));
    }
  }
  return dist;
}

// Whether the index's rows allow sq_exact_vec.
__device__ __forceinline__ bool sq_rows_vectorizable(const SqIndexView& ix) {
  if (ix.dim % 16 != 0) return false;
  const int ca = ix.l1_bits == 4 ? 8 : 16;
  if (ix.l1_code_bytes % ca != 0 || (reinterpret_cast<uintptr_t>(ix.l1) % ca) != 0) return false;
  if (!ix.residual) return true;
  const int ra = ix.residual_bits == 4 ? 8 : 16;
  return ix.rcb % ra == 0 && (reinterpret_cast<uintptr_t>(ix.residual) % ra) == 0 &&
         (reinterpret_cast<uintptr_t>(ix.qparams) % 8) == 0;
}

__device__ __forceinline__ float sq_exact_fast(const SqIndexView& ix, const float* q, int32_t id, bool vec) {
  return vec ? sq_exact_vec(ix, q, id) : sq_exact(ix, q, id);
}

// sq_exact of one candidate per group of 8 lanes (4 candidates per warp
// step), for rows sq_exact_vec can read and dim % 128 == 0.  Each lane
// squares 16 of every 128 dimensions; the sum then runs through the group's
// lanes in dimension order (lane k adds its 16 squares, then hands the
// partial sum to lane k + 1), so the FP32 additions are sq_exact's, in its
// order.  All 32 lanes must call it; every lane of a group returns the sum.
__device__ __forceinline__ float sq_exact_group(const SqIndexView& ix, const float* q, int32_t id, int lane) {
  const int sub = lane & 7, leader = lane & ~7;
  const uint8_t* l1 = ix.l1 + static_cast<size_t>(id) * ix.l1_code_bytes;
  const uint8_t* res = ix.residual ? ix.residual + static_cast<size_t>(id) * ix.rcb : nullptr;
  const bool c4 = ix.l1_bits == 4, r4 = ix.residual_bits == 4;
  float rs = 0.0f, rz = 0.0f, acc = 0.0f;
  if (res) {
    const float2 qp = __ldg(reinterpret_cast<const float2*>(ix.qparams) + id);
    rs = qp.x;
    rz = qp.y;
  }
  for (int r = 0; r < ix.dim; r += 128) {
    const int g = r + sub * 16;
    const uint4 cv = group_load(l1, c4, g);
    const uint4 rv = res ? group_load(res, r4, g) : make_uint4(0u, 0u, 0u, 0u);
    float sq[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      float value = fadd(fmul(u8f(group_code(cv, c4, j)), ix.l1_scale), ix.l1_zero);
      if (res) value = fadd(value, fadd(fmul(u8f(group_code(rv, r4, j)), rs), rz));
      const float diff = fsub(q[g + j], value);
      sq[j] = fmul(diff, diff);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (sub == k) {
#pragma unroll
        for (int j = 0; j < 16; ++j) acc = fadd(acc, sq[j]);
      }
      acc = __shfl_sync(kFullMask, acc, leader | k);
    }
  }
  return acc;
}

// First occurrence in lane order among lanes that hold the same id.
__device__ __forceinline__ bool first_of_equal(bool active, int32_t id, int lane) {
  const unsigned act = __ballot_sync(kFullMask, active);
  const unsigned same = __match_any_sync(kFullMask, active ? id : -2 - lane) & act;
  return active && (__ffs(same) - 1) == lane;
}

// Shared memory of one warp of sq_search_kernel_t: the query, its codes, the
// batch of scored candidates, then the pool's and the frontier's on-chip
// levels (SqSearchArgs::pool_split / front_split entries).
__host__ __device__ inline size_t sq_search_warp_smem(int dim, int pool_split, int front_split) {
  return static_cast<size_t>(((dim * 4) + 15) & ~15) + static_cast<size_t>((dim + 15) & ~15) + 32 * 8 +
         static_cast<size_t>(pool_split + front_split) * 8;
}

size_t sq_search_smem_per_warp(int dim, int pool_split, int front_split) {
  return sq_search_warp_smem(dim, pool_split, front_split);
}

// Four CTAs per SM: the shared-memory share the host gives a CTA when one
// per SM is not enough for the batch (sq_search_core) allows no more.
template <bool kSplit>
__global__ void __launch_bounds__(kSearchWarps * 32, 4)
sq_search_kernel_t(SqSearchArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const SqIndexView& ix = a.ix;
  const int qbytes = ((ix.dim * 4) + 15) & ~15;
  const int cbytes = ((ix.dim + 15) & ~15);
  uint8_t* base = smem + static_cast<size_t>(warp) * sq_search_warp_smem(ix.dim, a.pool_split, a.front_split);
  float* q = reinterpret_cast<float*>(base);
  uint8_t* qc = base + qbytes;
  HeapEntry* work = reinterpret_cast<HeapEntry*>(base + qbytes + cbytes);  // 32 scored candidates
  const int slot = blockIdx.x * kSearchWarps + warp;
  HeapEntry* gpool = reinterpret_cast<HeapEntry*>(a.heaps) +
                     static_cast<size_t>(slot) * (a.max_pool + a.frontier_cap);
  const SplitHeap pool{work + 32, gpool, a.pool_split};
  const SplitHeap front{work + 32 + a.pool_split, gpool + a.max_pool, a.front_split};
  VisitedTable vt;
  vt.slots = a.visited + static_cast<size_t>(slot) * (a.visited_mask + 1ull);
  vt.mask = a.visited_mask;
  const bool sqmd = a.mode == kSqModeSqmd;
  const bool db = a.mode == kSqModeDb;
  const bool split = kSplit && sqmd && a.correction;   // the host checks the index supports it
  const bool exact = (sqmd || db) && a.correction;
  const bool vec = sq_rows_vectorizable(ix);
  const bool group_rows = vec && ix.dim % 128 == 0;

  // Lane 0 applies the batch's scored candidates (work[0..cnt)) to the heaps
  // in batch order.  keep marks the ones that can enter the pool: a full
  // pool's worst only falls, so a candidate not below it at the start of the
  // batch stays out (the strict '<' of sqmd_common.c:51-80), and skipping it
  // changes nothing.
  auto apply = [&](unsigned keep, int& psize, int& fsize, int cap, int fcap, int32_t& st) {
    if (lane != 0) return;
    for (; keep; keep &= keep - 1u) {
      const int t = __ffs(keep) - 1;
      const HeapEntry c = work[t];
      if (pool_insert(pool, &psize, cap, c.id, c.dist)) {
        if (fsize < fcap) {
          front[fsize] = c;
          front_sift_up(front, fsize);
          ++fsize;
        } else if (!sqmd) {
          st = kStatusFrontierFull;
        }
      }
    }
  };
  // The keep mask of a batch: lanes holding a scored candidate (fresh) whose
  // distance may still enter the pool; each writes its entry at its rank.
  auto stage = [&](bool fresh, int32_t id, float d, int psize, int cap) -> unsigned {
    float worst = 0.0f;
    if (lane == 0 && psize > 0) worst = pool[0].dist;
    worst = __shfl_sync(kFullMask, worst, 0);
    const int ps = __shfl_sync(kFullMask, psize, 0);
    const bool keep = fresh && (ps < cap || d < worst);
    const unsigned km = __ballot_sync(kFullMask, keep);
    if (keep) work[__popc(km & ((1u << lane) - 1u))] = HeapEntry{id, d};
    __syncwarp();
    const int cnt = __popc(km);
    return cnt == 32 ? 0xffffffffu : (1u << cnt) - 1u;
  };

  for (;;) {
    int qi = 0;
    if (lane == 0) qi = static_cast<int>(atomicAdd(a.next_query, 1u));
    qi = __shfl_sync(kFullMask, qi, 0);
    if (qi >= a.nq) break;
    int32_t* status = a.status + qi;
    int cap = a.pool_sizes[qi];
    if (!sqmd && cap > 2000) cap = 2000;  // DSP_SEARCH_MAX_POOL
    const int expand = min(a.expand_count, ix.degree);
    if (cap <= 0 || cap > a.max_pool || expand <= 0 || a.entry_points <= 0 ||
        (sqmd && expand > 32) || (!sqmd && a.num_out <= 0)) {
      if (lane == 0) *status = kStatusBadParam;
      continue;
    }
    // frontier capacity the reference allocates for this request
    // (the DB-pair search grows its frontier up to n entries)
    const long long fcap_ref = db ? static_cast<long long>(ix.n)
                               : sqmd ? static_cast<long long>(a.entry_points) + static_cast<long long>(cap) * a.expand_count
                                      : static_cast<long long>(a.entry_points) + static_cast<long long>(cap) * expand;
    const int fcap = static_cast<int>(min(fcap_ref, static_cast<long long>(a.frontier_cap)));
    // query and its quantized codes (retrieval_quantize_query_u8/_u4,
    // l1_int8_core.c:13-63); with the split distance the codes of the
    // 17-fold refined grid instead (sq_split.cuh) and their sum
    const float inv = __frcp_rn(ix.l1_scale);
    const int levels = ix.l1_bits == 4 ? 15 : 255;
    const double step = split ? split_step(ix.l1_scale) : 0.0;
    unsigned long long sum_q = 0;
    bool qbad = false;
    for (int d = lane; d < ix.dim; d += kWarp) {
      const float v = a.queries[static_cast<size_t>(qi) * ix.dim + d];
      q[d] = v;
      if (split) {
        uint8_t c = 0;
        qbad |= !split_code(v, ix.l1_zero, step, &c);
        qc[d] = c;
        sum_q += c;
      } else {
        int c = static_cast<int>(roundf(fmul(fsub(v, ix.l1_zero), inv)));
        c = c < 0 ? 0 : (c > levels ? levels : c);
        qc[d] = static_cast<uint8_t>(c);
      }
    }
    if (split) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) sum_q += __shfl_xor_sync(kFullMask, sum_q, off);
      if (__any_sync(kFullMask, qbad)) {
        if (lane == 0) *status = kStatusNumeric;
        continue;
      }
    }
    __syncwarp();
    vt.gen = a.gen_base + static_cast<uint32_t>(qi);
    int psize = 0, fsize = 0;
    int32_t st = kStatusOk;
    unsigned long long scored = 0, turns = 0, dedup = 0;

    // ---- entries: the request's entry list (the host draws it once for all
    // queries, SqSearchArgs::entry_ids), claimed in list order
    for (int base_e = 0; base_e < a.entry_count && st == kStatusOk; base_e += kWarp) {
      const int e = base_e + lane;
      const bool active = e < a.entry_count;
      const int32_t id = active ? __ldg(a.entry_ids + e) : -1;
      bool fresh = false;
      // DSP: duplicates after the first are skipped; SQMD: the list holds
      // distinct ids (the reference's de-duplication) claimed here as
      // sqmd_cpu_state_seed does
      const bool first = sqmd ? active : first_of_equal(active, id, lane);
      if (first) {
        const int r = visited_insert(vt, static_cast<uint32_t>(id));
        if (r < 0) st = kStatusTableFull;
        fresh = r == 1;
      }
      float d = 0.0f;
      if (fresh) {
        // SQMD seeds carry the corrected distance (sqmd_make_seed); DSP and
        // DB-pair entries the coarse one (db_search_state_init)
        d = split ? split_seed_distance(ix, qc, sum_q, id, step)
                  : (sqmd && a.correction) ? sq_exact_fast(ix, q, id, vec) : sq_coarse(ix, qc, id);
        if (sqmd && a.correction && (!isfinite(d) || d < 0.0f)) st = kStatusNumeric;
      }
      if (__any_sync(kFullMask, st != kStatusOk)) { st = st != kStatusOk ? st : kStatusNumeric; break; }
      const unsigned keep = stage(fresh, id, d, psize, cap);
      apply(keep, psize, fsize, cap, fcap, st);
      st = __shfl_sync(kFullMask, st, 0);
      __syncwarp();
    }
    st = __shfl_sync(kFullMask, st, 0);

    // ---- expansion loop
    while (st == kStatusOk) {
      int32_t src = -1;
      if (lane == 0) {
        while (fsize > 0 && psize >= cap && front[0].dist > pool[0].dist) front_pop(front, &fsize);
        if (fsize > 0) src = front_pop(front, &fsize);
      }
      src = __shfl_sync(kFullMask, src, 0);
      if (src < 0) break;
      const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
      int nw = 0;
      for (int b = 0; b < expand; b += kWarp) {
        const int j = b + lane;
        int32_t nid = j < expand ? __ldg(row + j) : -1;
        bool ok = j < expand && nid >= 0 && nid < ix.n && (!sqmd || nid != src);
        const bool first = first_of_equal(ok, nid, lane);
        if (ok && !first) ++dedup;        // duplicate earlier in this row
        bool fresh = false;
        if (first) {
          const int r = visited_insert(vt, static_cast<uint32_t>(nid));
          if (r < 0) st = kStatusTableFull;
          fresh = r == 1;
          if (r == 0) ++dedup;
        }
        float d = 0.0f;
        bool dbad = false;
        if (fresh && split) {
          // sqmd_source_job_commit (sqmd_common.c:1533-1556): the lane's
          // coarse distance plus the host's delta, tiny negatives clamped
          const float dl = split_delta(ix, qc, sum_q, nid, step);
          d = split_sum(split_coarse(ix, qc, nid, step), dl);
          dbad = !isfinite(dl) || !isfinite(d) || d < 0.0f;
        } else if (exact && group_rows && __popc(__ballot_sync(kFullMask, fresh)) <= 8) {
          // few new neighbours (the usual case once the pool settles): a
          // group of 8 lanes per candidate instead of a lane each
          const unsigned fm = __ballot_sync(kFullMask, fresh);
          const int nf = __popc(fm);
          const int rank = __popc(fm & ((1u << lane) - 1u));
          if (fresh) work[rank].id = nid;     // the candidates in lane order
          __syncwarp();
          for (int t0 = 0; t0 < nf; t0 += 4) {
            const int t = t0 + (lane >> 3);
            const float gd = sq_exact_group(ix, q, t < nf ? work[t].id : 0, lane);
            const float mine = __shfl_sync(kFullMask, gd, ((rank - t0) & 3) * 8);
            if (fresh && rank >= t0 && rank < t0 + 4) d = mine;
          }
        } else if (fresh) {
          d = exact ? sq_exact_fast(ix, q, nid, vec) : sq_coarse(ix, qc, nid);
        }
        if (split && __any_sync(kFullMask, dbad)) { st = kStatusNumeric; break; }
        if (__any_sync(kFullMask, st != kStatusOk)) { st = kStatusTableFull; break; }
        nw += __popc(__ballot_sync(kFullMask, fresh));
        const unsigned keep = stage(fresh, nid, d, psize, cap);
        apply(keep, psize, fsize, cap, fcap, st);
        st = __shfl_sync(kFullMask, st, 0);
        __syncwarp();
        if (st != kStatusOk) break;
      }
      ++turns;
      scored += nw;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dedup += __shfl_xor_sync(kFullMask, dedup, off);
    if (st != kStatusOk) {
      if (lane == 0) *status = st;
      continue;
    }
    if (lane == 0) {
      // sqmd_heap_sort / dsp_heap_sort: in-place heap sort, ascending
      for (int i = psize - 1; i > 0; --i) {
        const HeapEntry t = pool[0];
        pool[0] = pool[i];
        pool[i] = t;
        pool_sift_down(pool, i, 0);
      }
    }
    // the heaps (and their sizes) are lane 0's: broadcast the pool size
    psize = __shfl_sync(kFullMask, psize, 0);
    __syncwarp();
    const int limit = sqmd ? a.out_stride : a.num_out;
    const int outn = min(psize, min(limit, a.out_stride));
    for (int i = lane; i < outn; i += kWarp) {
      const HeapEntry e = pool[i];
      a.out_ids[static_cast<size_t>(qi) * a.out_stride + i] = e.id;
      a.out_dists[static_cast<size_t>(qi) * a.out_stride + i] = e.dist;
    }
    if (lane == 0) {
      a.out_counts[qi] = outn;
      if (a.stats) {
        unsigned long long* s = a.stats + static_cast<size_t>(qi) * 4;
        s[0] = scored;
        s[1] = sqmd ? scored : 0ull;
        s[2] = turns;
        s[3] = dedup;
      }
    }
    __syncwarp();
  }
}


SqSearchFn sq_search_kernel_for(bool split) {
  return split ? sq_search_kernel_t<true> : sq_search_kernel_t<false>;
}

// ---------------------------------------------------------------------------
// DB-pair search, one step per launch (calculator_retrieval_search_db).  Warp
// w serves slot w when io.op[w] asks for it:
//   kDbInit   db_search_state_init (retrieval_async_dsp_search.c:1205-1301):
//             quantized query, cleared visited bitmap, entries (graph entry,
//             then the LCG of dsp_search_select_entry_id) with their coarse
//             distances inserted in draw order;
//   kDbStep   db_search_apply_corrections (:1371-1389) for the ids the last
//             step returned, with the corrected distances the caller wrote
//             into io.corr, then db_search_expand_one_step (:1303-1369): pop
//             (dropping entries worse than a full pool's worst), read up to
//             expand_limit neighbours, skip invalid and visited ids, and
//             return the rest with their coarse distances -- or finished;
//   kDbFinish dsp_heap_sort and the first num_out entries.
// Heap operations run on lane 0 in the reference's order; lanes compute the
// coarse distances.
__global__ void __launch_bounds__(kDbSlots * 32) db_step_kernel(DbArgs a) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  DbIo& io = *a.io;
  const int op = io.op[w];
  if (op == kDbNone) return;
  const SqIndexView& ix = a.ix;
  DbSlot& s = a.slots[w];
  HeapEntry* pool = reinterpret_cast<HeapEntry*>(a.pools) + static_cast<size_t>(w) * a.pool_cap;
  HeapEntry* front = reinterpret_cast<HeapEntry*>(a.fronts) + static_cast<size_t>(w) * a.frontier_cap;
  const size_t vwords = (static_cast<size_t>(ix.n) + 31) / 32;
  uint32_t* visited = a.visited + static_cast<size_t>(w) * vwords;
  __shared__ HeapEntry work[kDbSlots][32];
  __shared__ int32_t ids[kDbSlots][32];
  int st = kStatusOk;
  auto push = [&](int32_t id, float d) {   // lane 0: pool insert, then frontier push
    if (pool_insert(pool, &s.psize, a.pool_cap, id, d)) {
      if (s.fsize >= a.frontier_cap) { st = kStatusFrontierFull; return; }
      front[s.fsize] = HeapEntry{id, d};
      front_sift_up(front, s.fsize);
      ++s.fsize;
    }
  };
  auto test_and_set = [&](int32_t id) {     // lane 0 only
    uint32_t& word = visited[id >> 5];
    const uint32_t bit = 1u << (id & 31);
    const bool seen = (word & bit) != 0;
    word |= bit;
    return !seen;
  };
  if (op == kDbInit) {
    const float* q = a.queries + static_cast<size_t>(w) * ix.dim;
    const float inv = __frcp_rn(ix.l1_scale);
    const int levels = ix.l1_bits == 4 ? 15 : 255;
    for (int d = lane; d < ix.dim; d += kWarp) {
      int c = static_cast<int>(roundf(fmul(fsub(q[d], ix.l1_zero), inv)));
      s.qc[d] = static_cast<uint8_t>(c < 0 ? 0 : (c > levels ? levels : c));
    }
    for (size_t i = lane; i < vwords; i += kWarp) visited[i] = 0u;
    if (lane == 0) { s.psize = s.fsize = s.finished = s.last_count = 0; }
    __syncwarp();
    __threadfence_block();
    const int entries = min(a.entry_points, ix.n);
    uint32_t lcg = 42u;   // DSP_SEARCH_ENTRY_SEED
    for (int e0 = 0; e0 < entries && st == kStatusOk; e0 += kWarp) {
      if (lane == 0) {
        for (int t = 0; t < kWarp; ++t) {
          const int i = e0 + t;
          int32_t id = -1;
          if (i < entries) {
            if (i == 0 && a.graph_entry >= 0 && a.graph_entry < ix.n) {
              id = a.graph_entry;
            } else {
              lcg = lcg * 1103515245u + 12345u;
              id = static_cast<int32_t>((static_cast<uint64_t>(lcg) * static_cast<uint64_t>(ix.n)) >> 32);
            }
            if (!test_and_set(id)) id = -1;
          }
          ids[w][t] = id;
        }
      }
      __syncwarp();
      const int32_t id = ids[w][lane];
      work[w][lane] = HeapEntry{id, id >= 0 ? sq_coarse(ix, s.qc, id) : 0.0f};
      __syncwarp();
      if (lane == 0)
        for (int t = 0; t < kWarp && st == kStatusOk; ++t)
          if (work[w][t].id >= 0) push(work[w][t].id, work[w][t].dist);
      st = __shfl_sync(kFullMask, st, 0);
      __syncwarp();
    }
    if (lane == 0) io.status[w] = st;
    return;
  }
  if (op == kDbFinish) {
    if (lane == 0) {
      for (int i = s.psize - 1; i > 0; --i) {     // dsp_heap_sort
        const HeapEntry t = pool[0];
        pool[0] = pool[i];
        pool[i] = t;
        pool_sift_down(pool, i, 0);
      }
      const int outn = min(a.num_out, s.psize);
      for (int i = 0; i < outn; ++i) {
        a.out_ids[static_cast<size_t>(w) * a.num_out + i] = pool[i].id;
        a.out_dists[static_cast<size_t>(w) * a.num_out + i] = pool[i].dist;
      }
      io.out_count[w] = outn;
      io.status[w] = kStatusOk;
    }
    return;
  }
  // kDbStep: the caller's corrections of the last step, then the next step
  int32_t src = -1;
  if (lane == 0) {
    const int nc = s.last_count;
    for (int t = 0; t < nc && st == kStatusOk; ++t) push(s.last_ids[t], io.corr[w][t]);
    if (st == kStatusOk) {
      while (s.fsize > 0 && s.psize >= a.pool_cap && front[0].dist > pool[0].dist) front_pop(front, &s.fsize);
      if (s.fsize > 0) src = front_pop(front, &s.fsize);
    }
  }
  st = __shfl_sync(kFullMask, st, 0);
  src = __shfl_sync(kFullMask, src, 0);
  if (st != kStatusOk || src < 0) {
    if (lane == 0) {
      s.finished = src < 0 ? 1 : s.finished;
      s.last_count = 0;
      io.count[w] = 0;
      io.finished[w] = src < 0;
      io.status[w] = st;
    }
    return;
  }
  if (lane == 0) {
    const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
    int cnt = 0;
    for (int j = 0; j < a.expand_limit && cnt < kDbItems; ++j) {
      const int32_t nid = row[j];
      if (nid < 0 || nid >= ix.n) continue;
      if (!test_and_set(nid)) continue;
      ids[w][cnt++] = nid;
    }
    s.last_count = cnt;
    io.count[w] = cnt;
    io.finished[w] = 0;
    io.status[w] = kStatusOk;
  }
  __syncwarp();
  const int cnt = __shfl_sync(kFullMask, lane == 0 ? s.last_count : 0, 0);
  if (lane < cnt) {
    const int32_t nid = ids[w][lane];
    s.last_ids[lane] = nid;
    io.ids[w][lane] = nid;
    io.coarse[w][lane] = sq_coarse(ix, s.qc, nid);
  }
}

void launch_db_step(const DbArgs& a, cudaStream_t s) { db_step_kernel<<<1, kDbSlots * 32, 0, s>>>(a); }

}  // namespace rover
