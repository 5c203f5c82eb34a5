// pq_search.cu -- pure-PQ beam search on sm_100a, one warp per query.
//
// Semantics follow retrieval_pure_pq_search_scalar_with_policy
// (src/dsp_demo/retrieval_sqmd_pure_pq.c:793-969) with the ONLINE residual
// policy (retrieval_pq_residual_query_evaluate, retrieval_pq_residual.c:983)
// and the final refine (refine_impl, retrieval_final_refine.c:256-292).
//
// The reference keeps a bounded max-heap pool and a min-heap frontier under
// the strict total order (distance, id).  Because that order is total, the
// pool after any sequence of inserts is the top-L of everything scored, and
// the frontier pop that survives the pool-membership check is always the best
// not-yet-expanded pool entry.  The kernel therefore keeps the pool as a
// sorted list of 64-bit keys in shared memory with an "expanded" bit and
// expands the first unexpanded entry each step; this yields the same pool,
// the same expansion sequence and the same statistics as the heaps.
//
// Per expansion the warp reads the adjacency row, checks the valid-prefix
// rule (pure_pq_graph_row_count, :59-87), claims first visits in a per-warp
// visited table, scores the new neighbours (one lane each: ADC from the
// codebook in the reference's order plus the residual correction), sorts them
// with a warp bitonic network and merges them into the list.

#include "pq_common.cuh"

namespace rover {

// Score batch_ids[0..nb) (one lane per candidate) into keys[0..nb).
// Returns false when the reference would reject any candidate.
template <int M, int SUB, int RBITS>
__device__ __noinline__ bool score_batch(const PqSearchArgs& a, const float* q, const int32_t* batch_ids, int nb,
                                         uint64_t* keys, int lane) {
  bool bad = false;
  for (int e = lane; e < nb; e += kWarp) {
    const int32_t id = batch_ids[e];
    float adc, dist;
    if (score_one<M, SUB, RBITS>(a.ix, q, id, a.correction != 0, &adc, &dist)) keys[e] = make_key(dist, id);
    else bad = true;
  }
  __syncwarp();
  return !__any_sync(kFullMask, bad);
}

template <int M, int SUB, int RBITS>
__device__ bool score_and_merge(const PqSearchArgs& a, const float* q, uint64_t* list, int* size, int cap,
                                uint64_t* stage, const int32_t* batch_ids, int nb, int* cursor, int lane) {
  if (!score_batch<M, SUB, RBITS>(a, q, batch_ids, nb, stage, lane)) return false;
  merge_scored(list, size, cap, stage, nb, cursor, lane);
  return true;
}

template <int M, int SUB, int RBITS>
__global__ void __launch_bounds__(kSearchWarps * 32)
pq_search_kernel_t(PqSearchArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  uint8_t* base = smem + static_cast<size_t>(warp) * a.smem_per_warp;
  float* q = reinterpret_cast<float*>(base);
  uint64_t* list = reinterpret_cast<uint64_t*>(base + a.smem_query_bytes);
  uint64_t* stage = list + a.max_pool;                 // kMaxBatch keys
  int32_t* batch = reinterpret_cast<int32_t*>(stage + kMaxBatch);  // kMaxBatch ids
  const int slot = blockIdx.x * kSearchWarps + warp;
  VisitedTable vt;
  vt.slots = a.visited + static_cast<size_t>(slot) * (a.visited_mask + 1ull);
  vt.mask = a.visited_mask;
  const PqIndexView& ix = a.ix;

  for (;;) {
    int item = 0;
    if (lane == 0) item = static_cast<int>(atomicAdd(a.next_query, 1u));
    item = __shfl_sync(kFullMask, item, 0);
    if (item >= a.nq) break;
    const int qi = a.order ? __ldg(a.order + item) : item;

    const int cap = a.pool_sizes[qi];
    int32_t* status = a.status + qi;
    const int expand = min(a.expand_count, ix.degree);
    if (cap <= 0 || cap > a.max_pool || expand <= 0 || expand > kMaxBatch || a.entry_points <= 0) {
      if (lane == 0) *status = kStatusBadParam;
      continue;
    }
    for (int d = lane; d < ix.dim; d += kWarp) q[d] = a.queries[static_cast<size_t>(qi) * ix.dim + d];
    __syncwarp();
    // retrieval_pq_build_lut fails the query if any LUT entry is not finite
    // (built only when the bound of lut_provably_safe cannot exclude it)
    bool bad = false;
    const bool lut_safe = lut_provably_safe(ix, q, lane);
    for (int e = lut_safe ? ix.m * ix.ks : lane; e < ix.m * ix.ks; e += kWarp) {
      const int m = e / ix.ks;
      const float* cen = ix.codebook + static_cast<size_t>(e) * ix.subdim;
      float acc = 0.0f;
      for (int j = 0; j < ix.subdim; ++j) {
        const float diff = fsub(q[m * ix.subdim + j], __ldg(cen + j));
        acc = fadd(acc, fmul(diff, diff));
      }
      if (!isfinite(acc)) bad = true;
    }
    if (__any_sync(kFullMask, bad)) {
      if (lane == 0) *status = kStatusNumeric;
      continue;
    }
    vt.gen = (a.gen_dev ? *a.gen_dev : a.gen_base) + static_cast<uint32_t>(qi);
    int size = 0, cursor = 0;
    unsigned long long scored = 0, expanded = 0, dedup = 0;
    int32_t st = kStatusOk;
    const uint32_t load_limit = (a.visited_mask + 1u) >> 1;

    // entry ids: graph entry first, then the LCG of pure_pq_make_seed_ids
    // (retrieval_rpc_demo_pure_pq.c:192-208), processed in chunks of 32.
    const int entries = min(a.entry_points, ix.n);
    uint32_t lcg = a.seed;
    for (int base_e = 0; base_e < entries && st == kStatusOk; base_e += kWarp) {
      if (lane == 0) {
        for (int t = 0; t < kWarp && base_e + t < entries; ++t) {
          const int i = base_e + t;
          int32_t id;
          if (i == 0 && a.graph_entry >= 0 && a.graph_entry < ix.n) {
            id = a.graph_entry;
          } else {
            lcg = lcg * 1103515245u + 12345u;
            id = static_cast<int32_t>((static_cast<uint64_t>(lcg) * static_cast<uint64_t>(ix.n)) >> 32);
          }
          stage[t] = static_cast<uint64_t>(id);
        }
      }
      __syncwarp();
      const int e = base_e + lane;
      int fresh = 0;
      int32_t id = -1;
      if (e < entries) {
        id = static_cast<int32_t>(stage[lane]);
        const int r = visited_insert(vt, static_cast<uint32_t>(id));
        if (r < 0) st = kStatusTableFull;
        fresh = r == 1;
        if (r == 0) ++dedup;
      }
      __syncwarp();
      const unsigned fm = __ballot_sync(kFullMask, fresh);
      const int nb = __popc(fm);
      if (fresh) batch[__popc(fm & ((1u << lane) - 1u))] = id;
      __syncwarp();
      if (__any_sync(kFullMask, st != kStatusOk)) { st = kStatusTableFull; break; }
      scored += nb;
      if (nb > 0 && !score_and_merge<M, SUB, RBITS>(a, q, list, &size, cap, stage, batch, nb, &cursor, lane)) {
        st = kStatusNumeric;
        break;
      }
    }

    // expansion loop
    while (st == kStatusOk) {
      int pos = -1;
      for (int b = cursor & ~31; b < size; b += kWarp) {
        const int i = b + lane;
        const bool cand = i >= cursor && i < size && !(list[i] & kExpandedBit);
        const unsigned m = __ballot_sync(kFullMask, cand);
        if (m) { pos = b + __ffs(m) - 1; break; }
      }
      if (pos < 0) break;
      cursor = pos + 1;
      const int32_t src = key_id(list[pos]);
      __syncwarp();
      if (lane == 0) list[pos] |= kExpandedBit;
      const int32_t* row = ix.graph + static_cast<size_t>(src) * ix.degree;
      // valid-prefix rule (pure_pq_graph_row_count)
      int first_pad = expand;
      bool row_bad = false;
      for (int b = 0; b < expand; b += kWarp) {
        const int j = b + lane;
        const int32_t nid = j < expand ? __ldg(row + j) : -1;
        const unsigned pad = __ballot_sync(kFullMask, j < expand && nid == -1);
        if (pad && first_pad == expand) first_pad = b + __ffs(pad) - 1;
      }
      for (int b = 0; b < expand; b += kWarp) {
        const int j = b + lane;
        if (j < expand) {
          const int32_t nid = __ldg(row + j);
          if (j < first_pad) row_bad |= (nid < 0 || nid >= ix.n);
          else row_bad |= (nid != -1);
        }
      }
      if (__any_sync(kFullMask, row_bad)) { st = kStatusBadRow; break; }
      // first visits, in row order
      int nb = 0;
      bool full = false;
      for (int b = 0; b < first_pad; b += kWarp) {
        const int j = b + lane;
        int fresh = 0;
        int32_t nid = -1;
        if (j < first_pad) {
          nid = __ldg(row + j);
          const int r = visited_insert(vt, static_cast<uint32_t>(nid));
          full |= r < 0;
          fresh = r == 1;
          if (r == 0) ++dedup;
        }
        const unsigned fm = __ballot_sync(kFullMask, fresh);
        if (fresh) batch[nb + __popc(fm & ((1u << lane) - 1u))] = nid;
        nb += __popc(fm);
      }
      ++expanded;
      if (__any_sync(kFullMask, full) || scored + nb > load_limit) { st = kStatusTableFull; break; }
      __syncwarp();
      if (nb == 0) continue;
      scored += nb;
      if (!score_and_merge<M, SUB, RBITS>(a, q, list, &size, cap, stage, batch, nb, &cursor, lane)) {
        st = kStatusNumeric;
        break;
      }
    }

    // dedup counts were per lane: reduce
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dedup += __shfl_xor_sync(kFullMask, dedup, off);
    if (st != kStatusOk) {
      if (lane == 0) *status = st;
      continue;
    }
    __syncwarp();
    pq_finish_query(a, q, list, size, qi, lane, base, scored, a.correction ? scored : 0ull, expanded, dedup);
    __syncwarp();
  }
}

// Kernel instantiation for an index shape: Ks=256 shapes with a specialised
// scorer, the generic kernel otherwise.
PqSearchFn pq_search_kernel_for(const PqIndexView& ix, bool correction) {
  if (ix.ks == 256 && ix.code_bytes == ix.m) {
    const bool r8 = !correction || ix.residual_bits == 8;
    const bool r4 = correction && ix.residual_bits == 4;
    if (r8 || r4) {
#define ROVER_PQ_SHAPE(MM, SS)                                                 \
  if (ix.m == MM && ix.subdim == SS)                                           \
    return r8 ? pq_search_kernel_t<MM, SS, 8> : pq_search_kernel_t<MM, SS, 4>;
      ROVER_PQ_SHAPE(16, 8)
      ROVER_PQ_SHAPE(32, 4)
      ROVER_PQ_SHAPE(24, 4)
      ROVER_PQ_SHAPE(8, 8)
      ROVER_PQ_SHAPE(16, 4)
#undef ROVER_PQ_SHAPE
    }
  }
  return pq_search_kernel_t<0, 0, 0>;
}

}  // namespace rover
